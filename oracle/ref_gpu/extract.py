"""Build recipe for the reference's own GPU kernels (comparison arms only).

TEST INFRASTRUCTURE.  Reads the two CUDA source strings the reference
compiles with NVRTC at run time -- ``KERNEL_SRC`` (align_score_kernel) and
``KERNEL_H2_SRC`` (align_score_kernel_h2) in
crates/eschalign/src/cuda/kernel.rs -- where they lie in the reference tree,
and writes them, concatenated as the reference does for sm_80+
(cuda/mod.rs:386-397), to oracle/_ref/ref_kernels.cu.  The output stays under
oracle/_ref/ (git-ignored); nothing of the reference enters the repository.

    python oracle/ref_gpu/extract.py [REFERENCE_ROOT]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(os.path.dirname(HERE), "_ref")


def raw_string(src: str, name: str) -> str:
    m = re.search(r'const\s+' + name + r'\s*:\s*&str\s*=\s*r#"(.*?)"#;', src, re.S)
    if not m:
        raise SystemExit(f"{name} not found")
    return m.group(1)


def main(root: str) -> str:
    path = os.path.join(root, "crates/eschalign/src/cuda/kernel.rs")
    with open(path) as fh:
        src = fh.read()
    body = raw_string(src, "KERNEL_SRC") + raw_string(src, "KERNEL_H2_SRC")
    os.makedirs(OUT_DIR, exist_ok=True)
    out = os.path.join(OUT_DIR, "ref_kernels.cu")
    with open(out, "w") as fh:
        fh.write("// generated from crates/eschalign/src/cuda/kernel.rs (KERNEL_SRC + "
                 "KERNEL_H2_SRC); comparison arms only\n")
        fh.write(body)
    return out


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: extract.py <reference checkout>")
    print(main(sys.argv[1]))

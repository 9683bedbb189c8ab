/*
 * esg_pairs.c -- restatement of eschalign's paired-end scoring inputs.
 *
 * TEST INFRASTRUCTURE ONLY (see esg_oracle.h).  Placeholder unit; the pair
 * candidate ranking and adapter trimming are restated here.
 */
#include "esg_oracle.h"

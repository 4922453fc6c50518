/*
 * mom6_oracle_cc.c -- CPU restatements of the reference CUDA C kernels
 * (src/cuda_c/*.cu), one function per launch_* entry point, prefixed occ_.
 * TEST INFRASTRUCTURE ONLY (see mom6_oracle.h).
 */
#include "mom6_oracle.h"

/*
 * CPU oracle for the Vlasov-Poisson sweeps: C restatement of the reference's
 * PyTorch algorithm, built with OpenMP so it also serves as the multi-threaded
 * CPU baseline timed by bench.py.
 *
 * TEST INFRASTRUCTURE ONLY: the product (the CUDA library and its Python
 * mirror) never links, loads or calls this file. See vp_oracle_body.h for the
 * routines and the reference lines each one follows.
 */
#include <math.h>
#include <stdlib.h>
#include <stdint.h>

#define REAL double
#define SFX f64
#include "vp_oracle_body.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX f32
#include "vp_oracle_body.h"
#undef REAL
#undef SFX

#ifdef _OPENMP
#include <omp.h>
int or_num_threads(void) { return omp_get_max_threads(); }
void or_set_num_threads(int n) { omp_set_num_threads(n); }
#else
int or_num_threads(void) { return 1; }
void or_set_num_threads(int n) { (void)n; }
#endif

/*
 * hydist_oracle.h — CPU oracle for the GPU-hydist ADI hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a C restatement of the reference's FP64
 * kernels (UVZSolver_multithread.cu, support_funcs.cu, Sediment_Transport.cu,
 * constant.cuh) and of the launch sequence of Engine.py:144-366 / rep.py:126-139.
 * It is the parity checker for the CUDA library and the timed CPU baseline
 * ("port", OpenMP over grid lines).  Nothing in the product links or calls it.
 *
 * Parity pin: the restatement is checked bit-for-bit against the reference's own
 * kernel sources compiled and executed launch-for-launch by oracle/ref_harness.cpp
 * (CPU emulation build, and the sm_100a build on the GPU), see tests/test_oracle_pin.py.
 */
#ifndef HYDIST_ORACLE_H
#define HYDIST_ORACLE_H

#include <stddef.h>
#include "../include/hydist_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OraSim OraSim;

OraSim* ora_create(const HydCaseParams* p, int N, int M);
void ora_destroy(OraSim* s);

/* Direct pointer to an oracle field (same names and sizes as hyd_get_field);
 * *is_int is set to 1 for int32 fields.  NULL for an unknown name. */
void* ora_field(OraSim* s, const char* name, int* is_int, size_t* count);

int ora_set_boundary(OraSim* s, const int* boundary_type, const double* const* tables,
                     const double* const* cc, const int* nseg, int total_time);

/* rep.py:126-139 */
void ora_init(OraSim* s, double t_start);
/* rep.py:126-131 with pick_up: keeps the mask set before the call */
void ora_init_pickup(OraSim* s, double t_start);
/* Engine.py:144-366, nsteps iterations of the while loop */
void ora_step(OraSim* s, int nsteps);
double ora_time(const OraSim* s);
/* Resume support: set the time and the edge concentration scales (hmax_u, _d, _l, _r). */
void ora_set_time(OraSim* s, double t);
void ora_set_hmax(OraSim* s, const double* hmax4);
void ora_set_threads(int n);
/* Water account of the following steps into acc[0..4] (accumulated; null to stop): the
 * library's budget terms restated on the oracle's step (edge inflow, opened, closed, loss
 * to cells a sweep leaves unsolved, one-cell edge faces), m^3.  Not in the reference. */
void ora_water_enable(OraSim* s, double* acc);
/* Debug aid: print the first non-finite field value after each phase (stderr). */
void ora_set_trace(int on);

/* The reference's Thomas solver (UVZSolver_multithread.cu:203-228), for
 * known-answer tests of the tridiagonal path. */
void ora_tridiag(int sn, const double* AA, const double* BB, const double* CC, const double* DD,
                 double* x, double* Ap, double* Bp, double* ep);

/* Derived sediment constants evaluated as the reference's device helpers do
 * (constant.cuh:126-133): out[0]=Windx, out[1]=Windy, out[2]=Ufr, out[3]=Dxr, out[4]=wss. */
void ora_derived_constants(const HydCaseParams* p, double* out);

#ifdef __cplusplus
}
#endif
#endif

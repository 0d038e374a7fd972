/*
 * bd_oracle.h -- CPU restatement of bdsim's ChainIntegrator step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA integrator is compared
 * against: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it. The product (bdsim_b200/) never links or calls it.
 *
 * Pinned against (a) the golden vectors of the reference's own C++ tests
 * (tests/test_*.cpp, Fortran/MATLAB-derived), and (b) the reference C++
 * itself compiled from source into oracle/_ref/ (see oracle/Makefile).
 *
 * Parameters use the public layout of include/bdsim_cuda.h.
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H

#include <stdint.h>

#include "../include/bdsim_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Rng::ran_1 (src/rng.cpp:41-70) on state {ix, iy, seed}. */
void bdo_ran1(int32_t state[3], int n, double* out);

/* solve_implicit_r (src/spring.cpp:123-172): reduced length and force factor.
   Returns 0, or a BDCU_ST_* bit on failure. */
int bdo_solve_implicit_r(int spring_type, double dtby4, double gama, double natscl,
                         double* length, double* force_factor);

/* solve_connector (src/spring.cpp:174-181). */
int bdo_solve_connector(const double gamma[3], double dt, const bdcu_phys* p, double out[3]);

/* Per-bead forces at R (N x 3 row-major). arena: see bdsim_cuda.h. */
void bdo_spring_force(const double* R, int N, const bdcu_phys* p, double* F);
void bdo_bending_force(const double* R, int N, const bdcu_phys* p, double* F);
void bdo_ev_force(const double* R, int N, const bdcu_phys* p, const double* arena, double* F);
void bdo_external_force(int N, const bdcu_phys* p, const double* arena, double t, double* F);
/* spring + EV + bending (bindings/module.cpp:67-76) */
void bdo_total_force(const double* R, int N, const bdcu_phys* p, const double* arena, double* F);
void bdo_kappa(const bdcu_phys* p, const double* arena, double t, double K[9]);

/* Unit bonds (N-1 x 3) and bond cosines (N-2) (src/config.cpp:8-46). */
void bdo_unit_bonds_and_cosines(const double* R, int N, double* unit, double* cosines);

/* rpy_diffusion_matrix (src/hydrodynamics.cpp:12-54), n = 3N, row-major. */
void bdo_rpy_matrix(const double* R, int N, double hstar, double* D);
/* cholesky_lower (src/linalg.cpp:91-107). Returns 0 or BDCU_ST_NOT_PD. */
int bdo_cholesky(const double* D, int n, double* L);
/* spectral_bounds (src/hydrodynamics.cpp:224-264) with an optional warm-start
   cache (cache_vec length n, *cache_valid flag). */
void bdo_spectral_bounds(const double* D, int n, double* cache_vec, int* cache_valid,
                         double* lmin, double* lmax, int* steps_out);
/* chebyshev_sqrt_times (src/hydrodynamics.cpp:317-337). x0, out: n. */
void bdo_chebyshev_sqrt_times(const double* D, int n, const double* x0, double mult,
                              double fd_tol, double* cache_vec, int* cache_valid,
                              double* out, int* nterms, double* fd_err);

/* time_integrate_chain (src/integrator.cpp:174-177): integrate R (N x 3) in
   place over sim's [time_start, time_end]. rng advanced in place.
   cache_vec/cache_valid: if NULL a fresh cache is used (the reference's
   per-call reset); else the given cache persists across calls.
   counters may be NULL. Returns a BDCU_ST_* bitmask (0 = clean). */
int bdo_integrate(double* R, const bdcu_phys* p, const bdcu_sim* s, const double* arena,
                  int32_t rng[3], double* cache_vec, int* cache_valid,
                  bdcu_counters* counters);

/* Many independent chains on `n_threads` host threads (pthreads). R is the
   concatenation of the chains' N x 3 blocks (bead_offset[c] = first bead of
   chain c). status: n_chains out. */
int bdo_integrate_many(double* R, const int64_t* bead_offset, int n_chains,
                       const bdcu_phys* p, const bdcu_sim* s, const double* arena,
                       int32_t* rng, int32_t* status, int n_threads);

#ifdef __cplusplus
}
#endif

#endif

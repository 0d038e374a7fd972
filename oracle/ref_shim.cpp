// ref_shim.cpp -- C entry points over the reference bdsim C++ core.
//
// TEST INFRASTRUCTURE ONLY. oracle/Makefile compiles this file together with
// the reference's own sources (src/*.cpp of the bdsim project, read in place,
// never copied) into oracle/_ref/libbdref.so. Tests use it to pin the C
// restatement (bd_oracle.c) and the CUDA integrator against the real
// reference; bench.py's reference arm times it on the host cores.
//
// Parameters arrive in the public layout of include/bdsim_cuda.h and are
// converted to the reference's PhysParams / SimParams here.
#include "config.hpp"
#include "excluded_volume.hpp"
#include "hydrodynamics.hpp"
#include "integrator.hpp"
#include "linalg.hpp"
#include "model.hpp"
#include "spring.hpp"

#include <cstring>
#include <exception>
#include <thread>
#include <atomic>
#include <vector>

#include "../include/bdsim_cuda.h"

using namespace bdsim;

namespace {

Vec3Field to_field(const double* R, int N) {
    Vec3Field f(N);
    for (int i = 0; i < N; ++i) f[i] = {R[3 * i], R[3 * i + 1], R[3 * i + 2]};
    return f;
}

void from_field(const Vec3Field& f, double* R) {
    for (size_t i = 0; i < f.size(); ++i)
        for (int d = 0; d < 3; ++d) R[3 * i + d] = f[i][d];
}

PhysParams to_phys(const bdcu_phys* p, const double* arena) {
    PhysParams q;
    q.number_of_beads = p->n_beads;
    q.spring.type = static_cast<Spring>(p->spring_type);
    q.spring.sqrtb = p->sqrtb;
    q.spring.natural_length = p->natural_length;
    q.ev.type = static_cast<EV>(p->ev_type);
    q.ev.zstar = p->zstar;
    q.ev.dstar = p->dstar;
    q.ev.min_cutoff = p->min_cutoff;
    q.ev.max_cutoff = p->max_cutoff;
    q.ev.contour_dist_for_EV = p->contour_dist_for_ev;
    if (p->phi_offset >= 0) {
        const size_t nn = static_cast<size_t>(p->n_beads) * p->n_beads;
        q.ev.phi.assign(arena + p->phi_offset, arena + p->phi_offset + nn);
    }
    q.bend.type = static_cast<Bending>(p->bend_type);
    q.bend.stiffness = p->bend_stiffness;
    if (p->flow_n_times == 0) {
        Mat3 K{};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) K[i][j] = p->flow_kappa[3 * i + j];
        q.flow = Flow::constant(K);
    } else {
        const int n = p->flow_n_times;
        const double* t = arena + p->flow_offset;
        std::vector<dp> times(t, t + n);
        std::vector<Mat3> Ks(n);
        for (int s = 0; s < n; ++s)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Ks[s][i][j] = t[n + 9 * s + 3 * i + j];
        q.flow = Flow::time_varying(times, Ks);
    }
    const double* e = arena + p->ext_offset;
    for (int k = 0; k < p->ext_n_entries; ++k) {
        const int bead = static_cast<int>(e[0]);
        const int n = static_cast<int>(e[5]);
        if (e[1] != 0.0) {
            q.external.add_constant(bead, Vec3{e[2], e[3], e[4]});
        } else {
            std::vector<dp> times(e + 6, e + 6 + n);
            std::vector<Vec3> vals(n);
            for (int j = 0; j < n; ++j) vals[j] = {e[6 + n + 3 * j], e[6 + n + 3 * j + 1], e[6 + n + 3 * j + 2]};
            q.external.add_time_varying(bead, times, vals);
        }
        e += 6 + 4 * n;
    }
    q.hstar = p->hstar;
    q.hi_method = static_cast<DelSMethod>(p->hi_method);
    q.ncheb_multiplier = p->ncheb_multiplier;
    q.fd_err_max = p->fd_err_max;
    q.equilibration = p->equilibration != 0;
    return q;
}

SimParams to_sim(const bdcu_sim* s) {
    SimParams q;
    q.time_start = s->time_start;
    q.time_end = s->time_end;
    q.dt = s->dt;
    q.implicit_loop_tol = s->implicit_loop_tol;
    q.update_center_of_mass = s->update_center_of_mass != 0;
    return q;
}

Matrix to_matrix(const double* D, int n) {
    Matrix M(n);
    std::memcpy(M.a.data(), D, sizeof(double) * static_cast<size_t>(n) * n);
    return M;
}

}  // namespace

extern "C" {

void ref_ran1(int32_t state[3], int n, double* out) {
    Rng r;
    r.restore({state[0], state[1], state[2]});
    r.ran_1(n, out);
    const Rng::State s = r.save();
    state[0] = s.ix;
    state[1] = s.iy;
    state[2] = s.seed;
}

void ref_solve_implicit_r(int type, double dtby4, double gama, double natscl, double* length, double* ff) {
    const SpringSolution s = solve_implicit_r(static_cast<Spring>(type), dtby4, gama, natscl);
    *length = s.length;
    *ff = s.force_factor;
}

void ref_solve_connector(const double gamma[3], double dt, const bdcu_phys* p, double out[3]) {
    SpringParams sp{static_cast<Spring>(p->spring_type), p->sqrtb, p->natural_length};
    const Vec3 q = solve_connector(Vec3{gamma[0], gamma[1], gamma[2]}, dt, sp);
    for (int d = 0; d < 3; ++d) out[d] = q[d];
}

void ref_total_force(const double* R, int N, const bdcu_phys* p, const double* arena, double* F) {
    PhysParams phys = to_phys(p, arena);
    phys.number_of_beads = N;
    PhysicalModel model(phys);
    const Vec3Field Rf = to_field(R, N);
    const ChainGeometry g = chain_geometry(Rf);
    Vec3Field f = spring_force(g, model.spring());
    const Vec3Field fe = model.non_spring_force({Rf, g});
    for (size_t i = 0; i < f.size(); ++i) f[i] = f[i] + fe[i];
    from_field(f, F);
}

void ref_rpy_matrix(const double* R, int N, double hstar, double* D) {
    const Matrix M = rpy_diffusion_matrix(to_field(R, N), hstar);
    std::memcpy(D, M.a.data(), sizeof(double) * M.a.size());
}

int ref_cholesky(const double* D, int n, double* L) {
    try {
        const Matrix M = cholesky_lower(to_matrix(D, n));
        std::memcpy(L, M.a.data(), sizeof(double) * M.a.size());
        return 0;
    } catch (const std::exception&) {
        return BDCU_ST_NOT_PD;
    }
}

void ref_spectral_bounds(const double* D, int n, double* cache_vec, int* cache_valid, double* lmin,
                         double* lmax) {
    SpectralCache cache;
    if (cache_vec && *cache_valid) cache.start.assign(cache_vec, cache_vec + n);
    const auto b = spectral_bounds(to_matrix(D, n), cache_vec ? &cache : nullptr);
    *lmin = b.first;
    *lmax = b.second;
    if (cache_vec) {
        *cache_valid = static_cast<int>(cache.start.size()) == n;
        if (*cache_valid) std::memcpy(cache_vec, cache.start.data(), sizeof(double) * n);
    }
}

void ref_chebyshev_sqrt_times(const double* D, int n, const double* x0, double mult, double fd_tol,
                              double* out, int* nterms, double* fd_err) {
    const ChebyshevResult r = chebyshev_sqrt_times(to_matrix(D, n), to_field(x0, n / 3), mult, fd_tol, nullptr);
    from_field(r.value, out);
    *nterms = r.nterms;
    *fd_err = r.fd_error;
}

// time_integrate_chain with a fresh model (cold spectral cache), exactly the
// reference call. Returns 0, or BDCU_ST_NOT_PD if the reference threw.
int ref_integrate(double* R, const bdcu_phys* p, const bdcu_sim* s, const double* arena, int32_t rng[3]) {
    PhysParams phys = to_phys(p, arena);
    const SimParams sim = to_sim(s);
    Vec3Field Rf = to_field(R, p->n_beads);
    phys.number_of_beads = p->n_beads;
    Rng r;
    r.restore({rng[0], rng[1], rng[2]});
    try {
        time_integrate_chain(Rf, phys, sim, r);
    } catch (const std::exception&) {
        return BDCU_ST_NOT_PD;
    }
    from_field(Rf, R);
    const Rng::State st = r.save();
    rng[0] = st.ix;
    rng[1] = st.iy;
    rng[2] = st.seed;
    return 0;
}

// Many chains on n_threads std::threads, each owning disjoint chains (the
// reference's process-pool parallelism, parallel.py:62-93, without Python).
int ref_integrate_many(double* R, const int64_t* bead_offset, int n_chains, const bdcu_phys* p,
                       const bdcu_sim* s, const double* arena, int32_t* rng, int32_t* status,
                       int n_threads) {
    if (n_threads < 1) n_threads = 1;
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t)
        pool.emplace_back([&]() {
            for (;;) {
                const int c = next.fetch_add(1);
                if (c >= n_chains) break;
                status[c] = ref_integrate(R + 3 * bead_offset[c], &p[c], &s[c], arena, rng + 3 * c);
            }
        });
    for (auto& th : pool) th.join();
    return 0;
}

}  // extern "C"

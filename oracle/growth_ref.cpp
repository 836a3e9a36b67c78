// C ABI over the reference's own C++ forward solver (include/morphompm/
// growth_solver.h, used unmodified from the reference tree), so that tests and
// the benchmark's CPU arm can run it from Python.  Test and measurement
// infrastructure only: nothing in the product links it.
//
// The solver is the reference's FP32 forward oracle: node-centred quadratic
// MLS-MPM, Hencky-Kirchhoff stress through its one-sided Jacobi SVD with the
// singular values clamped at 1e-6, separate force grid, mass threshold 1e-9,
// gravity, per-step damping, always-advected positions
// (growth_solver.h:82-221, math/svd.h:18-108).
#include <cstring>
#include <new>

#include "morphompm/growth_solver.h"

using morphompm::GrowthSolver;
using morphompm::math::Matrix3;
using morphompm::math::Vec3;

extern "C" {

void* ref_create(int N, float dx, float E, float nu, float damping, float gx, float gy, float gz) {
    GrowthSolver* s = new (std::nothrow) GrowthSolver(N, dx);
    if (!s) return nullptr;
    s->set_material(E, nu);
    s->set_damping(damping);
    s->set_gravity(Vec3(gx, gy, gz));
    return s;
}

void ref_destroy(void* h) { delete static_cast<GrowthSolver*>(h); }

// n particles at x (n x 3), each of the given mass and density (vol0 = mass / density)
void ref_add(void* h, long long n, const float* x, float mass, float density) {
    GrowthSolver* s = static_cast<GrowthSolver*>(h);
    for (long long p = 0; p < n; ++p) s->add_particle(Vec3(x[3 * p], x[3 * p + 1], x[3 * p + 2]), mass, density);
}

// n particles, each with its own mass and density (vol0 = mass / density)
void ref_add_each(void* h, long long n, const float* x, const float* mass, const float* density) {
    GrowthSolver* s = static_cast<GrowthSolver*>(h);
    for (long long p = 0; p < n; ++p)
        s->add_particle(Vec3(x[3 * p], x[3 * p + 1], x[3 * p + 2]), mass[p], density[p]);
}

// Fg = g I for every particle
void ref_set_growth(void* h, float g) {
    for (auto& p : static_cast<GrowthSolver*>(h)->particles()) p.Fg = Matrix3::scale(g, g, g);
}

// per-particle growth tensors, Fg (n x 3 x 3, row-major)
void ref_set_growth_tensors(void* h, const float* Fg) {
    auto& ps = static_cast<GrowthSolver*>(h)->particles();
    for (size_t p = 0; p < ps.size(); ++p)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) ps[p].Fg.m[i][j] = Fg[9 * p + 3 * i + j];
}

void ref_step(void* h, float dt, int steps) {
    GrowthSolver* s = static_cast<GrowthSolver*>(h);
    for (int t = 0; t < steps; ++t) s->step(dt);
}

// x, v (n x 3) and F, C (n x 3 x 3, row-major); any pointer may be null
void ref_get(void* h, float* x, float* v, float* F, float* C) {
    const auto& ps = static_cast<GrowthSolver*>(h)->particles();
    for (size_t p = 0; p < ps.size(); ++p) {
        const auto& q = ps[p];
        if (x) { x[3 * p] = q.x.x; x[3 * p + 1] = q.x.y; x[3 * p + 2] = q.x.z; }
        if (v) { v[3 * p] = q.v.x; v[3 * p + 1] = q.v.y; v[3 * p + 2] = q.v.z; }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                if (F) F[9 * p + 3 * i + j] = q.F.m[i][j];
                if (C) C[9 * p + 3 * i + j] = q.C.m[i][j];
            }
    }
}

}  // extern "C"

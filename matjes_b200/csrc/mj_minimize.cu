// Energy minimisation drivers on the device: the two routines of
// solvers/minimize.F90.
//
// mj_minimize (minimize_run, :57-166): velocity projection on the damping
// force F = B - (m.B) m (vector_utils/vector.f90:146-161).  Per iteration one
// field evaluation (any plan: stencil, ELL, dipolar) and two elementwise
// passes: k_vpo_force (F, the velocity update of euler_minimization and the two
// global sums V.F and |F|^2, reduced deterministically) and k_vpo_move (the
// projected velocity and the norm-keeping euler_o2_minimization move,
// solvers/solver.f90:129-160, with the largest |F| as the torque).  A device
// flag stops the iterations once the torque is below the criterion; the host
// looks at it every `check_every` iterations.
//
// mj_minimize_infdamp (minimize_infdamp_run, :169-258): every spin turned onto
// its normalised local field.  The reference visits the sites in order, each
// with the field of the current neighbours; here the sites are visited colour
// by colour with the colouring (x mod cx) + cx ((y mod cy) + cy (z mod cz)),
// chosen so that no coupling joins two sites of one colour: within a colour the
// updates are independent and run in parallel.  Single-atom stencil plans
// without the dipolar term.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "mj_device.cuh"
#include "mj_internal.hpp"
#include "mj_stencil.cuh"

namespace mj {
namespace {

struct MinState {
    double sums[2];                 // V.F and |F|^2 of the iteration
    unsigned long long maxt_bits;   // largest torque of the iteration (non-negative double bits)
    double last_maxt;               // torque of the last completed iteration
    long long iters;                // completed iterations
    int done;                       // converged
    int bad;                        // a site had a field shorter than 1e-8
};

__device__ __forceinline__ void max_torque(unsigned long long* bits, double t) {
    atomicMax(bits, static_cast<unsigned long long>(__double_as_longlong(t)));
}

// first predictor: F = B - (m.B) m, m <- F dt^2/(2 mass) + m (not normalised), V = 0
__global__ void k_vpo_init(int64_t N, double* __restrict__ m, const double* __restrict__ B, double* __restrict__ force,
                           double* __restrict__ vel, double dt, double mass) {
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    const double3 mi = ld3(m, i, N), b = ld3(B, i, N);
    const double d = dot(mi, b);
    const double3 F = make_double3(-(mi.x * d - b.x), -(mi.y * d - b.y), -(mi.z * d - b.z));
    st3(force, i, N, F);
    const double dt2 = dt * dt, m2 = mass * 2.0;
    st3(m, i, N, make_double3(F.x * dt2 / m2 + mi.x, F.y * dt2 / m2 + mi.y, F.z * dt2 / m2 + mi.z));
    st3(vel, i, N, make_double3(0.0, 0.0, 0.0));
}

__global__ void __launch_bounds__(256) k_vpo_force(int64_t N, const double* __restrict__ m, const double* __restrict__ B,
                                                   double* __restrict__ force, double* __restrict__ vel, double dt,
                                                   double mass, double* partials, unsigned int* counter, MinState* S,
                                                   int nblocks) {
    if (S->done) return;
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < N) {
        const double3 mi = ld3(m, i, N), b = ld3(B, i, N);
        const double d = dot(mi, b);
        const double3 F = make_double3(-(mi.x * d - b.x), -(mi.y * d - b.y), -(mi.z * d - b.z));
        const double3 f0 = ld3(force, i, N), v0 = ld3(vel, i, N);
        const double3 V = make_double3((f0.x + F.x) / 2.0 * dt / mass + v0.x, (f0.y + F.y) / 2.0 * dt / mass + v0.y,
                                       (f0.z + F.z) / 2.0 * dt / mass + v0.z);
        st3(force, i, N, F);
        st3(vel, i, N, V);
        v[0] = dot(V, F);
        v[1] = dot(F, F);
    }
    grid_reduce<2>(v, partials, counter, S->sums, nblocks);
}

__global__ void __launch_bounds__(256) k_vpo_move(int64_t N, double* __restrict__ m, const double* __restrict__ force,
                                                  double* __restrict__ vel, double dt, double mass, MinState* S) {
    if (S->done) return;
    const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i >= N) return;
    const double dumy = S->sums[0], fn = S->sums[1];
    const double3 F = ld3(force, i, N);
    const double3 v = fabs(dumy) > 1e-8 ? make_double3(dumy * F.x / fn, dumy * F.y / fn, dumy * F.z / fn)
                                        : make_double3(0.0, 0.0, 0.0);
    st3(vel, i, N, v);
    const double3 mi = ld3(m, i, N);
    const double c = dt * dt;
    const double3 s = make_double3(F.x * c / mass / 2.0 + v.x * dt + mi.x, F.y * c / mass / 2.0 + v.y * dt + mi.y,
                                   F.z * c / mass / 2.0 + v.z * dt + mi.z);
    const double ni = sqrt(dot(mi, mi)), nf = sqrt(dot(s, s));
    st3(m, i, N, nf > 1e-8 ? make_double3(s.x / nf * ni, s.y / nf * ni, s.z / nf * ni) : make_double3(0.0, 0.0, 0.0));
    max_torque(&S->maxt_bits, sqrt(dot(F, F)));
}

// end of an iteration: count it, keep its torque, stop below the criterion
__global__ void k_min_check(MinState* S, double conv_torque) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || S->done) return;
    S->iters += 1;
    const double mt = __longlong_as_double(static_cast<long long>(S->maxt_bits));
    S->last_maxt = mt;
    if (mt < conv_torque) S->done = 1;
    S->maxt_bits = 0ull;
}

// one colour of the infinite-damping sweep
__global__ void __launch_bounds__(256) k_infdamp(const __grid_constant__ StencilParams P, const double* __restrict__ bmap,
                                                 double* m, int cx, int cy, int cz, int col, MinState* S) {
    if (S->done) return;
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
    if (x >= P.L[0] || y >= P.L[1]) return;
    if ((x % cx) + cx * ((y % cy) + cy * (z % cz)) != col) return;
    const int64_t N = static_cast<int64_t>(P.L[0]) * P.L[1] * P.L[2];
    const int64_t i = x + static_cast<int64_t>(P.L[0]) * (y + static_cast<int64_t>(P.L[1]) * z);
    const double3 m0 = ld3(m, i, N);
    const double3 B = add3(w_apply(P, m, N, x, y, z, m0), zeeman(P, bmap, i, N));
    const double bn = sqrt(dot(B, B));
    if (bn < 1e-8) {
        atomicOr(&S->bad, 1);
        return;
    }
    const double3 Bh = make_double3(B.x / bn, B.y / bn, B.z / bn);
    const double3 t = cross(m0, Bh);
    max_torque(&S->maxt_bits, fmax(fabs(t.x), fmax(fabs(t.y), fabs(t.z))));
    if (sqrt(dot(m0, m0)) > 1e-8) st3(m, i, N, Bh);
}

// smallest colouring (cx, cy, cz) in which no stencil offset joins two sites of one colour
bool choose_colors(const StencilParams& sp, int c[3]) {
    int best = 1 << 30;
    for (int cz = 1; cz <= 4; ++cz)
        for (int cy = 1; cy <= 4; ++cy)
            for (int cx = 1; cx <= 4; ++cx) {
                const int cc[3] = {cx, cy, cz};
                bool ok = cx * cy * cz < best;
                for (int d = 0; d < 3 && ok; ++d)
                    if (sp.periodic[d] && sp.L[d] % cc[d] != 0) ok = false;
                for (int k = 0; k < sp.n_off && ok; ++k) {
                    bool differs = false;
                    for (int d = 0; d < 3; ++d) differs = differs || (((sp.off[k][d] % cc[d]) + cc[d]) % cc[d]) != 0;
                    if (!differs) ok = false;
                }
                if (ok) {
                    best = cx * cy * cz;
                    c[0] = cx;
                    c[1] = cy;
                    c[2] = cz;
                }
            }
    return best < (1 << 30);
}

mj_status read_state(MinState* d_S, int64_t* iterations, double* torque, cudaStream_t s, MinState* h) {
    mj_status st = cuda_status(cudaMemcpyAsync(h, d_S, sizeof(MinState), cudaMemcpyDeviceToHost, s), "minimiser state");
    if (st != MJ_OK) return st;
    if ((st = cuda_status(cudaStreamSynchronize(s), "minimiser")) != MJ_OK) return st;
    if (iterations) *iterations = h->iters;
    if (torque) *torque = h->last_maxt;
    return MJ_OK;
}

}  // namespace
}  // namespace mj

using namespace mj;

extern "C" {

mj_status mj_minimize(mj_plan* plan, double* m, const mj_min_params* p, int64_t max_iter, int64_t* iterations,
                      double* torque, void* stream) {
    if (!plan || !m || !p || max_iter < 0) return set_error(MJ_ERR_ARG, "bad minimisation arguments");
    if (!(p->mass != 0.0) || !(p->timestep > 0.0)) return set_error(MJ_ERR_ARG, "mass must be non-zero, timestep > 0");
    cudaSetDevice(plan->device);
    const int64_t N = plan->N;
    const size_t f3 = sizeof(double) * 3 * static_cast<size_t>(N);
    mj_status st;
    if (!plan->d_field && (st = cuda_status(cudaMalloc(&plan->d_field, f3), "field scratch")) != MJ_OK) return st;
    MinState* d_S = nullptr;
    if ((st = cuda_status(cudaMalloc(&d_S, sizeof(MinState)), "minimiser state")) != MJ_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* B = plan->d_field;
    double* force = plan->d_aux;
    double* vel = plan->d_aux2;
    const int nb = static_cast<int>((N + 255) / 256);
    const int check = std::max<int32_t>(1, p->check_every);
    MinState h{};
    cudaMemsetAsync(d_S, 0, sizeof(MinState), s);
    st = launch_field(plan, m, B, nullptr, nullptr, s);
    if (st == MJ_OK) {
        k_vpo_init<<<nb, 256, 0, s>>>(N, m, B, force, vel, p->timestep, p->mass);
        st = cuda_status(cudaGetLastError(), "k_vpo_init");
    }
    for (int64_t it = 0; st == MJ_OK && it < max_iter; ++it) {
        if ((st = launch_field(plan, m, B, nullptr, nullptr, s)) != MJ_OK) break;
        k_vpo_force<<<nb, 256, 0, s>>>(N, m, B, force, vel, p->timestep, p->mass, plan->d_partials, plan->d_counter, d_S,
                                       nb);
        k_vpo_move<<<nb, 256, 0, s>>>(N, m, force, vel, p->timestep, p->mass, d_S);
        k_min_check<<<1, 32, 0, s>>>(d_S, p->conv_torque);
        if ((st = cuda_status(cudaGetLastError(), "minimisation")) != MJ_OK) break;
        if ((it + 1) % check == 0 || it + 1 == max_iter) {
            if ((st = read_state(d_S, iterations, torque, s, &h)) != MJ_OK) break;
            if (h.done) break;
        }
    }
    if (st == MJ_OK && max_iter == 0) st = read_state(d_S, iterations, torque, s, &h);
    cudaFree(d_S);
    return st;
}

mj_status mj_minimize_infdamp(mj_plan* plan, double* m, const mj_min_params* p, int64_t max_iter, int64_t* iterations,
                              double* torque, int32_t* colors, void* stream) {
    if (!plan || !m || !p || max_iter < 0) return set_error(MJ_ERR_ARG, "bad minimisation arguments");
    if (!plan->is_stencil || plan->dip_on)
        return set_error(MJ_ERR_UNSUPPORTED, "the infinite-damping sweep needs a single-atom stencil plan, no dipolar term");
    int c[3] = {1, 1, 1};
    if (!choose_colors(plan->sp, c))
        return set_error(MJ_ERR_UNSUPPORTED, "no colouring of at most 4 x 4 x 4 fits the stencil and periodic sizes");
    if (colors)
        for (int d = 0; d < 3; ++d) colors[d] = c[d];
    cudaSetDevice(plan->device);
    mj_status st;
    MinState* d_S = nullptr;
    if ((st = cuda_status(cudaMalloc(&d_S, sizeof(MinState)), "minimiser state")) != MJ_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 grid((plan->sp.L[0] + 31) / 32, (plan->sp.L[1] + 7) / 8, plan->sp.L[2]), blk(32, 8);
    const int check = std::max<int32_t>(1, p->check_every);
    const int ncol = c[0] * c[1] * c[2];
    MinState h{};
    cudaMemsetAsync(d_S, 0, sizeof(MinState), s);
    for (int64_t it = 0; it < max_iter; ++it) {
        for (int col = 0; col < ncol; ++col)
            k_infdamp<<<grid, blk, 0, s>>>(plan->sp, plan->d_bmap, m, c[0], c[1], c[2], col, d_S);
        k_min_check<<<1, 32, 0, s>>>(d_S, p->conv_torque);
        if ((st = cuda_status(cudaGetLastError(), "infinite-damping sweep")) != MJ_OK) break;
        if ((it + 1) % check == 0 || it + 1 == max_iter) {
            if ((st = read_state(d_S, iterations, torque, s, &h)) != MJ_OK) break;
            if (h.bad) {
                st = set_error(MJ_ERR_ARG, "a site has an effective field shorter than 1e-8");
                break;
            }
            if (h.done) break;
        }
    }
    if (st == MJ_OK && max_iter == 0) st = read_state(d_S, iterations, torque, s, &h);
    cudaFree(d_S);
    return st;
}

}  // extern "C"

// Lanczos vector kernels.
//
// Reference: groundStateLieb.c:217-344 (lanczos) runs, per step i,
//   beta_i = |r|; v_{i+1} = r / beta_i; r = H v_{i+1} - beta_i v_i;
//   alpha_{i+1} = <v_{i+1}, r>; r -= alpha_{i+1} v_{i+1};
//   c_j = <v_j, r> (j <= i+1); r -= sum_j c_j v_j          (classical Gram-Schmidt)
// with a breakdown exit when beta_i / max(beta) < 1e-15 (returning i), all in
// FP64 complex on the host (serial dots, OpenMP update).
//
// Here every scalar stays on the device (alpha, beta, the breakdown flag and the
// reorthogonalisation coefficients live in a small state block), so a whole
// solve is a fixed launch sequence with no host round trip: it can be captured
// in a CUDA graph, and once the flag is set every later kernel returns at entry.
// Reductions go through per-block partials summed in block order by a single
// block, so results are bitwise reproducible run to run. The two passes of the
// reorthogonalisation read the Krylov basis once each (HBM bound, the dominant
// Lanczos cost beside H.psi): pass 1 stages a 1024-row slice of
// x = r - alpha v_{i+1} in shared memory and lets each warp stream one basis
// vector over it; pass 2 updates r row by row in the reference's per-element
// order (x - v_0 c_0 - v_1 c_1 - ...) and emits the norm partials of the next
// step.
#include <cuda_runtime.h>
#include "kernels.h"

namespace mcpi {

namespace {

constexpr int kThreads = 256;
constexpr int kParts = 592;          // blocks of the fixed-size reductions (4 x 148 SMs)
constexpr int kSlice = 1024;         // rows per block in reorthogonalisation pass 1

__device__ __forceinline__ double2 cmulc(double2 a, double2 b)  // conj(a) * b
{
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ double2 warp_sum(double2 v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Block-wide sum in a fixed order; result valid in thread 0.
__device__ __forceinline__ double2 block_sum(double2 v)
{
    __shared__ double2 red[kThreads / 32];
    v = warp_sum(v);
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x / 32); ++k) {
            r.x += red[k].x;
            r.y += red[k].y;
        }
    return r;
}

__device__ __forceinline__ bool stopped(const int *done) { return done && *done; }

// partial[b] = sum over the block's grid-stride rows of conj(a) b
__global__ void k_dot_partial(const double2 *__restrict__ a, const double2 *__restrict__ b,
                              int64_t n, double2 *__restrict__ partial, const int *done)
{
    if (stopped(done)) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * kThreads) {
        const double2 p = cmulc(a[r], b[r]);
        acc.x += p.x;
        acc.y += p.y;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// out = sum_b partial[b] (b in order); one block.
__global__ void k_sum_partials(const double2 *__restrict__ partial, int n, double2 *out,
                               const int *done)
{
    if (stopped(done)) return;
    double2 acc = make_double2(0.0, 0.0);
    // fixed assignment: thread t sums t, t+256, ... then a fixed-order block sum
    for (int b = threadIdx.x; b < n; b += kThreads) {
        acc.x += partial[b].x;
        acc.y += partial[b].y;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc;
}

// r -= beta_i v_prev ; partial of <v_cur, r>
__global__ void k_axpy_dot(const double2 *__restrict__ vprev, const double2 *__restrict__ vcur,
                           double2 *__restrict__ r, int64_t n, const double *beta_i,
                           double2 *__restrict__ partial, const int *done)
{
    if (stopped(done)) return;
    const double b = *beta_i;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        double2 y = r[x];
        const double2 p = vprev[x];
        y.x -= b * p.x;
        y.y -= b * p.y;
        r[x] = y;
        const double2 d = cmulc(vcur[x], y);
        acc.x += d.x;
        acc.y += d.y;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// r -= beta_i v_prev (the update of k_axpy_dot without its dot product)
__global__ void k_axpy(const double2 *__restrict__ vprev, double2 *__restrict__ r, int64_t n,
                       const double *beta_i, const int *done)
{
    if (stopped(done)) return;
    const double b = *beta_i;
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        double2 y = r[x];
        const double2 p = vprev[x];
        y.x -= b * p.x;
        y.y -= b * p.y;
        r[x] = y;
    }
}

// Pass 1: partial[j * nblk + b] = sum_{rows of slice b} conj(V_j) (r - alpha vcur)
__global__ void __launch_bounds__(kThreads) k_multidot(const double2 *__restrict__ V, int nvec,
                                                       int64_t n, const double2 *__restrict__ r,
                                                       const double2 *__restrict__ vcur,
                                                       const double2 *alpha,
                                                       double2 *__restrict__ partial,
                                                       const int *done)
{
    if (stopped(done)) return;
    __shared__ double2 xs[kSlice];
    const int64_t r0 = (int64_t)blockIdx.x * kSlice;
    const int rows = (int)((n - r0) < kSlice ? (n - r0) : kSlice);
    const double2 a = *alpha;
    for (int t = threadIdx.x; t < rows; t += kThreads) {
        const double2 y = r[r0 + t], v = vcur[r0 + t];
        // x = r - alpha * v (complex product as in the reference)
        xs[t] = make_double2(y.x - (a.x * v.x - a.y * v.y), y.y - (a.x * v.y + a.y * v.x));
    }
    __syncthreads();
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int j = w; j < nvec; j += kThreads / 32) {
        const double2 *vj = V + (size_t)j * n + r0;
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
        for (int t = lane; t < rows; t += 32) {
            const double2 p = cmulc(vj[t], xs[t]);
            acc.x += p.x;
            acc.y += p.y;
        }
        acc = warp_sum(acc);
        if (lane == 0) partial[(size_t)j * gridDim.x + blockIdx.x] = acc;
    }
}

// coef[j] = sum_b partial[j * nblk + b]; one warp per j, fixed order.
__global__ void k_multidot_finish(const double2 *__restrict__ partial, int nblk, int nvec,
                                  double2 *__restrict__ coef, const int *done)
{
    if (stopped(done)) return;
    const int j = blockIdx.x * (kThreads / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
    if (j >= nvec) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int b = lane; b < nblk; b += 32) {
        acc.x += partial[(size_t)j * nblk + b].x;
        acc.y += partial[(size_t)j * nblk + b].y;
    }
    acc = warp_sum(acc);
    if (lane == 0) coef[j] = acc;
}

constexpr int kUpdBatch = 8;   // basis entries in flight per thread in k_update

// Pass 2: r = (r - alpha vcur) - sum_j V_j coef_j ; partial of |r|^2
__global__ void __launch_bounds__(kThreads) k_update(const double2 *__restrict__ V, int nvec,
                                                     int64_t n, double2 *__restrict__ r,
                                                     const double2 *__restrict__ vcur,
                                                     const double2 *alpha,
                                                     const double2 *__restrict__ coef,
                                                     double2 *__restrict__ partial,
                                                     const int *done)
{
    if (stopped(done)) return;
    extern __shared__ double2 cs[];
    for (int j = threadIdx.x; j < nvec; j += kThreads) cs[j] = coef[j];
    __syncthreads();
    const double2 a = *alpha;
    double acc = 0.0;
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        const double2 y = r[x], v = vcur[x];
        double2 u = make_double2(y.x - (a.x * v.x - a.y * v.y), y.y - (a.x * v.y + a.y * v.x));
        // kUpdBatch basis entries loaded together, then subtracted in order j
        int j = 0;
        for (; j + kUpdBatch <= nvec; j += kUpdBatch) {
            double2 p[kUpdBatch];
#pragma unroll
            for (int q = 0; q < kUpdBatch; ++q) p[q] = V[(size_t)(j + q) * n + x];
#pragma unroll
            for (int q = 0; q < kUpdBatch; ++q) {
                const double2 c = cs[j + q];
                u.x -= p[q].x * c.x - p[q].y * c.y;
                u.y -= p[q].x * c.y + p[q].y * c.x;
            }
        }
        for (; j < nvec; ++j) {
            const double2 p = V[(size_t)j * n + x], c = cs[j];
            u.x -= p.x * c.x - p.y * c.y;
            u.y -= p.x * c.y + p.y * c.x;
        }
        r[x] = u;
        acc += u.x * u.x + u.y * u.y;
    }
    double2 s = block_sum(make_double2(acc, 0.0));
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// beta_i = sqrt(sum partials); breakdown test of groundStateLieb.c:287-292.
__global__ void k_beta(const double2 *__restrict__ partial, int n, int i, double tol,
                       double *beta, double *maxbeta, int *done, int *iters)
{
    if (*done) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < n; b += kThreads) acc.x += partial[b].x;
    acc = block_sum(acc);
    if (threadIdx.x == 0) {
        const double bi = sqrt(acc.x);
        beta[i] = bi;
        if (*maxbeta < bi) *maxbeta = bi;
        // a zero residual (or a zero maximum) is a breakdown too
        if (!(bi / *maxbeta >= tol)) {
            *done = 1;
            *iters = i;
        }
    }
}

// The same test from a norm^2 already summed over the ranks of a sharded solve.
__global__ void k_beta_total(const double *norm2, int i, double tol, double *beta, double *maxbeta, int *done,
                             int *iters)
{
    if (*done || threadIdx.x != 0) return;
    const double bi = sqrt(*norm2);
    beta[i] = bi;
    if (*maxbeta < bi) *maxbeta = bi;
    if (!(bi / *maxbeta >= tol)) {
        *done = 1;
        *iters = i;
    }
}

// *out = real part of sum_b partial[b] (b in order); one block.
__global__ void k_sum_partials_re(const double2 *__restrict__ partial, int n, double *out, const int *done)
{
    if (stopped(done)) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int b = threadIdx.x; b < n; b += kThreads) acc.x += partial[b].x;
    acc = block_sum(acc);
    if (threadIdx.x == 0) *out = acc.x;
}

__global__ void k_scale(const double2 *__restrict__ r, double2 *__restrict__ vnext, int64_t n,
                        const double *beta_i, const int *done)
{
    if (stopped(done)) return;
    const double b = *beta_i;
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        const double2 y = r[x];
        vnext[x] = make_double2(y.x / b, y.y / b);
    }
}

// acc (+)= z * v, z real (read from device memory); first = 1 overwrites acc.
__global__ void k_axpy_real(double2 *__restrict__ acc, const double2 *__restrict__ v, int64_t n,
                            const double *z, int first, const int *done)
{
    if (stopped(done)) return;
    const double c = *z;
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        const double2 p = v[x];
        double2 a = first ? make_double2(0.0, 0.0) : acc[x];
        a.x += p.x * c;
        a.y += p.y * c;
        acc[x] = a;
    }
}

// out = sum_k V_k z_k (groundStateLieb.c:454-458), z real.
__global__ void k_combine(const double2 *__restrict__ V, int nvec, int64_t n,
                          const double *__restrict__ z, double2 *__restrict__ out)
{
    extern __shared__ double zs[];
    for (int j = threadIdx.x; j < nvec; j += kThreads) zs[j] = z[j];
    __syncthreads();
    for (int64_t x = blockIdx.x * (int64_t)kThreads + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * kThreads) {
        double2 acc = make_double2(0.0, 0.0);
        for (int j = 0; j < nvec; ++j) {
            const double2 p = V[(size_t)j * n + x];
            acc.x += p.x * zs[j];
            acc.y += p.y * zs[j];
        }
        out[x] = acc;
    }
}

}  // namespace

static unsigned grid_for(int64_t n)
{
    int64_t g = (n + kThreads - 1) / kThreads;
    return (unsigned)(g < kParts ? (g > 0 ? g : 1) : kParts);
}

int lanczos_parts(int64_t nc)
{
    return (int)grid_for(nc);
}

size_t lanczos_partial_elems(int64_t nc, int lm)
{
    const size_t nblk = (size_t)((nc + kSlice - 1) / kSlice);
    const size_t a = (size_t)kParts, b = nblk * (size_t)(lm + 1);
    return a > b ? a : b;
}

cudaError_t launch_dot(const double2 *a, const double2 *b, int64_t nc, double2 *partial,
                       double2 *result, cudaStream_t st)
{
    const unsigned g = grid_for(nc);
    k_dot_partial<<<g, kThreads, 0, st>>>(a, b, nc, partial, nullptr);
    k_sum_partials<<<1, kThreads, 0, st>>>(partial, g, result, nullptr);
    return cudaGetLastError();
}

// r = H v0 on entry: alpha_0 = <v0, r>; r -= alpha_0 v0; norm partials.
cudaError_t launch_lanczos_start(const double2 *v0, const double2 *hv, double2 *r, int64_t nc,
                                 LanczosState s, cudaStream_t st)
{
    const unsigned g = grid_for(nc);
    if (hv != r) {
        cudaError_t e = cudaMemcpyAsync(r, hv, sizeof(double2) * nc, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
    }
    k_dot_partial<<<g, kThreads, 0, st>>>(v0, r, nc, s.partial, s.done);
    k_sum_partials<<<1, kThreads, 0, st>>>(s.partial, g, s.alpha, s.done);
    k_update<<<g, kThreads, 0, st>>>(nullptr, 0, nc, r, v0, s.alpha, nullptr, s.partial, s.done);
    return cudaGetLastError();
}

cudaError_t launch_lanczos_beta(int i, int lm, double tol, LanczosState s, cudaStream_t st)
{
    (void)lm;
    k_beta<<<1, kThreads, 0, st>>>(s.partial, s.nparts, i, tol, s.beta, s.maxbeta, s.done, s.iters);
    return cudaGetLastError();
}

cudaError_t launch_lanczos_scale(const double2 *r, double2 *vnext, int64_t nc, int i,
                                 LanczosState s, cudaStream_t st)
{
    k_scale<<<grid_for(nc), kThreads, 0, st>>>(r, vnext, nc, s.beta + i, s.done);
    return cudaGetLastError();
}

// r -= beta_i v_i ; alpha_{i+1} = <v_{i+1}, r>
cudaError_t launch_lanczos_alpha(const double2 *vprev, const double2 *vcur, double2 *r,
                                 int64_t nc, int i, LanczosState s, cudaStream_t st)
{
    const unsigned g = grid_for(nc);
    k_axpy_dot<<<g, kThreads, 0, st>>>(vprev, vcur, r, nc, s.beta + i, s.partial, s.done);
    k_sum_partials<<<1, kThreads, 0, st>>>(s.partial, g, s.alpha + i + 1, s.done);
    return cudaGetLastError();
}

// c_j = <V_j, r - alpha_{i+1} v_{i+1}>, j < nvec ; r = r - alpha v - sum c_j V_j ; norm partials
cudaError_t launch_lanczos_reorth(const double2 *V, int nvec, double2 *r, int64_t nc, int i,
                                  LanczosState s, cudaStream_t st)
{
    const double2 *vcur = V + (size_t)(i + 1) * nc;
    const unsigned nblk = (unsigned)((nc + kSlice - 1) / kSlice);
    k_multidot<<<nblk, kThreads, 0, st>>>(V, nvec, nc, r, vcur, s.alpha + i + 1, s.partial, s.done);
    k_multidot_finish<<<(nvec + 7) / 8, kThreads, 0, st>>>(s.partial, nblk, nvec, s.coef, s.done);
    const unsigned g = grid_for(nc);
    k_update<<<g, kThreads, sizeof(double2) * nvec, st>>>(V, nvec, nc, r, vcur, s.alpha + i + 1,
                                                         s.coef, s.partial, s.done);
    return cudaGetLastError();
}

// r -= alpha_{i+1} v_{i+1} ; norm partials (the step without reorthogonalisation)
cudaError_t launch_lanczos_no_reorth(const double2 *vcur, double2 *r, int64_t nc, int i, LanczosState s,
                                     cudaStream_t st)
{
    k_update<<<grid_for(nc), kThreads, 0, st>>>(nullptr, 0, nc, r, vcur, s.alpha + i + 1, nullptr, s.partial,
                                                s.done);
    return cudaGetLastError();
}

cudaError_t launch_lanczos_axpy(const double2 *vprev, double2 *r, int64_t nc, int i, LanczosState s,
                               cudaStream_t st)
{
    k_axpy<<<grid_for(nc), kThreads, 0, st>>>(vprev, r, nc, s.beta + i, s.done);
    return cudaGetLastError();
}

cudaError_t launch_axpy_real(double2 *acc, const double2 *v, int64_t nc, const double *z, int first,
                             cudaStream_t st)
{
    k_axpy_real<<<grid_for(nc), kThreads, 0, st>>>(acc, v, nc, z, first, nullptr);
    return cudaGetLastError();
}

// ---- row-shard primitives (one rank's rows of a sharded solve) --------------------

size_t shard_scratch_elems(int64_t n, int lm) { return lanczos_partial_elems(n, lm); }

cudaError_t launch_shard_scale(int64_t n, const double2 *r, double2 *vnext, const double *beta_i, const int *done,
                               cudaStream_t st)
{
    k_scale<<<grid_for(n), kThreads, 0, st>>>(r, vnext, n, beta_i, done);
    return cudaGetLastError();
}

cudaError_t launch_shard_axpy_dot(int64_t n, const double2 *vprev, const double2 *vcur, double2 *r,
                                  const double *beta_i, double2 *scratch, double2 *dot, const int *done,
                                  cudaStream_t st)
{
    const unsigned g = grid_for(n);
    if (vprev)
        k_axpy_dot<<<g, kThreads, 0, st>>>(vprev, vcur, r, n, beta_i, scratch, done);
    else
        k_dot_partial<<<g, kThreads, 0, st>>>(vcur, r, n, scratch, done);
    k_sum_partials<<<1, kThreads, 0, st>>>(scratch, g, dot, done);
    return cudaGetLastError();
}

cudaError_t launch_shard_multidot(int64_t n, const double2 *V, int nvec, const double2 *r, const double2 *vcur,
                                  const double2 *alpha, double2 *scratch, double2 *coef, const int *done,
                                  cudaStream_t st)
{
    const unsigned nblk = (unsigned)((n + kSlice - 1) / kSlice);
    k_multidot<<<nblk ? nblk : 1, kThreads, 0, st>>>(V, nvec, n, r, vcur, alpha, scratch, done);
    k_multidot_finish<<<(nvec + 7) / 8, kThreads, 0, st>>>(scratch, nblk, nvec, coef, done);
    return cudaGetLastError();
}

cudaError_t launch_shard_update(int64_t n, const double2 *V, int nvec, double2 *r, const double2 *vcur,
                                const double2 *alpha, const double2 *coef, double2 *scratch, double *norm2,
                                const int *done, cudaStream_t st)
{
    const unsigned g = grid_for(n);
    k_update<<<g, kThreads, sizeof(double2) * (nvec > 0 ? nvec : 0), st>>>(V, nvec, n, r, vcur, alpha, coef,
                                                                        scratch, done);
    k_sum_partials_re<<<1, kThreads, 0, st>>>(scratch, g, norm2, done);
    return cudaGetLastError();
}

cudaError_t launch_shard_beta(int i, double tol, const double *norm2, double *beta, double *maxbeta, int *done,
                              int *iters, cudaStream_t st)
{
    k_beta_total<<<1, 32, 0, st>>>(norm2, i, tol, beta, maxbeta, done, iters);
    return cudaGetLastError();
}

cudaError_t launch_combine(const double2 *V, int nvec, int64_t nc, const double *z,
                           double2 *out, cudaStream_t st)
{
    k_combine<<<grid_for(nc), kThreads, sizeof(double) * nvec, st>>>(V, nvec, nc, z, out);
    return cudaGetLastError();
}

}  // namespace mcpi

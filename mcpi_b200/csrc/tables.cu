// Reference-layout Fock tables, built on the device.
//
// The hot kernels need none of these (they hash on the fly, fock.cuh); they
// exist so that a caller of the reference interface gets bit-identical arrays:
//   IF      configurationsMap.h:309-344  IF[j + i*M] = occupation of orbital j
//   Map     configurationsMap.h:348-417  Map[i + k*nc + l*M*nc] = index of v-e_k+e_l, -1 if v_k=0
//   MapOT   configurationsMap.h:617-762  chunk per orbital with v_k >= 2,
//           MapOT[stride[i] + c*M^2 + (l + q*M)] = index of v - 2e_k + e_l + e_q
//   MapTT   configurationsMap.h:421-613  chunk per occupied pair k<s,
//           MapTT[stride[i] + c*M^2 + (l + q*M)] = index of v - e_k - e_s + e_l + e_q
// One thread per configuration decodes its row once and writes every entry it
// owns; strides are an exclusive scan (CUB) of the per-row chunk counts, kept in
// 64 bits here and narrowed to the reference's int32 only by the drop-in layer.
#include <cub/device/device_scan.cuh>
#include <cuda_runtime.h>
#include "fock.cuh"
#include "kernels.h"

namespace mcpi {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void load_w(const Space &sp, const SpaceTables &tb, uint32_t *W)
{
    for (int x = threadIdx.x; x < (sp.M - 1) * sp.wstride; x += blockDim.x) W[x] = tb.W[x];
    __syncthreads();
}

template <int M>
__global__ void k_focks(Space sp, SpaceTables tb, int32_t *__restrict__ IF)
{
    extern __shared__ uint32_t W[];
    load_w(sp, tb, W);
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= sp.nc) return;
    int v[M], P[M];
    decode<M>(i, sp.N, sp.nc, W, sp.wstride, v, P);
#pragma unroll
    for (int j = 0; j < M; ++j) IF[(size_t)i * M + j] = v[j];
}

// Packed occupations (bits per orbital) of every configuration, for kernels
// that would otherwise decode their row index.
template <int M>
__global__ void k_pack_occ(Space sp, SpaceTables tb, int bits, uint64_t *__restrict__ occ)
{
    extern __shared__ uint32_t W[];
    load_w(sp, tb, W);
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= sp.nc) return;
    int v[M], P[M];
    decode<M>(i, sp.N, sp.nc, W, sp.wstride, v, P);
    uint64_t w = 0;
#pragma unroll
    for (int j = 0; j < M; ++j) w |= (uint64_t)v[j] << (bits * j);
    occ[i] = w;
}

template <int M>
__global__ void k_one_one(Space sp, SpaceTables tb, int32_t *__restrict__ Map)
{
    extern __shared__ uint32_t W[];
    load_w(sp, tb, W);
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= sp.nc) return;
    const int ws = sp.wstride;
    int v[M], P[M];
    decode<M>(i, sp.N, sp.nc, W, ws, v, P);
    uint32_t A0[M], Am1[M], Ap1[M];
    prefix_table<M>(P, 0, W, ws, A0);
    prefix_table<M>(P, -1, W, ws, Am1);
    prefix_table<M>(P, 1, W, ws, Ap1);
    const size_t nc = sp.nc;
#pragma unroll
    for (int k = 0; k < M; ++k)
#pragma unroll
        for (int l = 0; l < M; ++l) {
            const int32_t val = v[k] < 1 ? -1 : (int32_t)idx_move1(sp.nc, A0, Am1, Ap1, k, l, M);
            Map[i + k * nc + (size_t)l * M * nc] = val;
        }
}

template <int M>
__device__ __forceinline__ int row_chunks(const int *v, int two_orbital)
{
    int c = 0;
    if (!two_orbital) {
#pragma unroll
        for (int k = 0; k < M; ++k) c += (v[k] >= 2);
    } else {
        int occ = 0;
#pragma unroll
        for (int k = 0; k < M; ++k) occ += (v[k] >= 1);
        c = occ * (occ - 1) / 2;
    }
    return c;
}

template <int M>
__global__ void k_chunk_counts(Space sp, SpaceTables tb, int two_orbital, int64_t *__restrict__ cnt)
{
    extern __shared__ uint32_t W[];
    load_w(sp, tb, W);
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= sp.nc) return;
    int v[M], P[M];
    decode<M>(i, sp.N, sp.nc, W, sp.wstride, v, P);
    cnt[i] = (int64_t)row_chunks<M>(v, two_orbital) * (M * M);
}

// Index of the N-configuration with prefix counts Pn (direct sum, O(M)).
template <int M>
__device__ __forceinline__ uint32_t index_of(const int *Pn, uint32_t nc, const uint32_t *W, int ws)
{
    uint32_t s = 0;
#pragma unroll
    for (int t = 0; t < M - 1; ++t) s += W[t * ws + Pn[t]];
    return nc - 1u - s;
}

template <int M>
__global__ void k_two_map(Space sp, SpaceTables tb, int two_orbital,
                          const int64_t *__restrict__ stride, int32_t *__restrict__ Map)
{
    extern __shared__ uint32_t W[];
    load_w(sp, tb, W);
    const uint32_t i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= sp.nc) return;
    const int ws = sp.wstride;
    int v[M], P[M];
    decode<M>(i, sp.N, sp.nc, W, ws, v, P);
    int64_t base = stride[i];
#pragma unroll 1
    for (int k = 0; k < M; ++k) {
        if (two_orbital ? (v[k] < 1) : (v[k] < 2)) continue;
#pragma unroll 1
        for (int s = two_orbital ? k + 1 : k; s < (two_orbital ? M : k + 1); ++s) {
            if (two_orbital && v[s] < 1) continue;
            // prefix counts of the (N-2)-configuration v - e_k - e_s
            int Q[M];
#pragma unroll
            for (int t = 0; t < M; ++t) Q[t] = P[t] - (t >= k) - (t >= s);
#pragma unroll 1
            for (int l = 0; l < M; ++l)
#pragma unroll 1
                for (int q = 0; q < M; ++q) {
                    int Pn[M];
#pragma unroll
                    for (int t = 0; t < M; ++t) Pn[t] = Q[t] + (t >= l) + (t >= q);
                    Map[base + l + q * M] = (int32_t)index_of<M>(Pn, sp.nc, W, ws);
                }
            base += M * M;
        }
    }
}

__global__ void k_total(const int64_t *stride, const int64_t *cnt, int64_t nc, int M, int64_t *total)
{
    *total = (stride[nc - 1] + cnt[nc - 1]) / ((int64_t)M * M);
}

__global__ void k_narrow(const int64_t *__restrict__ in, int32_t *__restrict__ out, int64_t n)
{
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n;
         x += (int64_t)gridDim.x * blockDim.x)
        out[x] = (int32_t)in[x];
}

size_t wbytes(const Space &sp) { return sizeof(uint32_t) * (sp.M > 1 ? (sp.M - 1) * sp.wstride : 1); }
unsigned gridn(const Space &sp) { return (sp.nc + kThreads - 1) / kThreads; }

template <template <int> class F, typename... A>
cudaError_t by_m(int M, A... a)
{
    switch (M) {
#define MCPI_CASE(m) \
    case m: return F<m>::run(a...);
        MCPI_CASE(1) MCPI_CASE(2) MCPI_CASE(3) MCPI_CASE(4) MCPI_CASE(5) MCPI_CASE(6)
        MCPI_CASE(7) MCPI_CASE(8) MCPI_CASE(9) MCPI_CASE(10) MCPI_CASE(11) MCPI_CASE(12)
        MCPI_CASE(13) MCPI_CASE(14) MCPI_CASE(15) MCPI_CASE(16)
#undef MCPI_CASE
    default: return cudaErrorInvalidValue;
    }
}

template <int M>
struct RunFocks {
    static cudaError_t run(Space sp, SpaceTables tb, int32_t *IF, cudaStream_t st)
    {
        k_focks<M><<<gridn(sp), kThreads, wbytes(sp), st>>>(sp, tb, IF);
        return cudaGetLastError();
    }
};

template <int M>
struct RunPackOcc {
    static cudaError_t run(Space sp, SpaceTables tb, int bits, uint64_t *occ, cudaStream_t st)
    {
        k_pack_occ<M><<<gridn(sp), kThreads, wbytes(sp), st>>>(sp, tb, bits, occ);
        return cudaGetLastError();
    }
};

template <int M>
struct RunOneOne {
    static cudaError_t run(Space sp, SpaceTables tb, int32_t *Map, cudaStream_t st)
    {
        k_one_one<M><<<gridn(sp), kThreads, wbytes(sp), st>>>(sp, tb, Map);
        return cudaGetLastError();
    }
};

template <int M>
struct RunCounts {
    static cudaError_t run(Space sp, SpaceTables tb, int two, int64_t *cnt, cudaStream_t st)
    {
        k_chunk_counts<M><<<gridn(sp), kThreads, wbytes(sp), st>>>(sp, tb, two, cnt);
        return cudaGetLastError();
    }
};

template <int M>
struct RunTwoMap {
    static cudaError_t run(Space sp, SpaceTables tb, int two, const int64_t *stride, int32_t *Map,
                           cudaStream_t st)
    {
        k_two_map<M><<<gridn(sp), kThreads, wbytes(sp), st>>>(sp, tb, two, stride, Map);
        return cudaGetLastError();
    }
};

}  // namespace

cudaError_t launch_focks(const Space &sp, const SpaceTables &tb, int32_t *IF, cudaStream_t st)
{
    return by_m<RunFocks>(sp.M, sp, tb, IF, st);
}

int occ_bits_for(int N, int M)
{
    int b = 1;
    while ((1 << b) <= N) ++b;
    return M * b <= 64 ? b : 0;
}

cudaError_t launch_pack_occ(const Space &sp, const SpaceTables &tb, uint64_t *occ, int bits, cudaStream_t st)
{
    if (bits <= 0 || sp.M * bits > 64) return cudaErrorInvalidValue;
    return by_m<RunPackOcc>(sp.M, sp, tb, bits, occ, st);
}

cudaError_t launch_one_one_map(const Space &sp, const SpaceTables &tb, int32_t *Map, cudaStream_t st)
{
    return by_m<RunOneOne>(sp.M, sp, tb, Map, st);
}

cudaError_t launch_chunk_counts(const Space &sp, const SpaceTables &tb, int two_orbital,
                                int64_t *counts, cudaStream_t st)
{
    return by_m<RunCounts>(sp.M, sp, tb, two_orbital, counts, st);
}

cudaError_t launch_stride_scan(const Space &sp, const int64_t *counts, int64_t *stride,
                               int64_t *d_total, void *scratch, size_t scratch_bytes,
                               size_t *scratch_needed, cudaStream_t st)
{
    size_t need = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, counts, stride, (int64_t)sp.nc, st);
    if (e != cudaSuccess) return e;
    if (scratch_needed) *scratch_needed = need;
    if (!scratch) return cudaSuccess;
    if (scratch_bytes < need) return cudaErrorInvalidValue;
    e = cub::DeviceScan::ExclusiveSum(scratch, need, counts, stride, (int64_t)sp.nc, st);
    if (e != cudaSuccess) return e;
    k_total<<<1, 1, 0, st>>>(stride, counts, (int64_t)sp.nc, sp.M, d_total);
    return cudaGetLastError();
}

cudaError_t launch_two_map(const Space &sp, const SpaceTables &tb, int two_orbital,
                           const int64_t *stride, int32_t *Map, cudaStream_t st)
{
    return by_m<RunTwoMap>(sp.M, sp, tb, two_orbital, stride, Map, st);
}

cudaError_t launch_narrow_stride(const int64_t *in, int32_t *out, int64_t n, cudaStream_t st)
{
    k_narrow<<<592, 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

}  // namespace mcpi

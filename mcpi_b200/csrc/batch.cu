// Batched Lanczos: many ground-state solves of different (N, M) advanced
// together in one device arena and replayed as one CUDA graph.
//
// Reference: groundStateLieb.c runs one solve at a time (lanczos :217-344,
// ground :348-471) with host dots and a host tridiagonal solve. Here every
// member keeps the reference's recurrence (full classical Gram-Schmidt
// reorthogonalisation, breakdown at beta_i / max beta < 1e-15) but each
// stage is one launch over all members:
//   * H.psi: per orbital count M one launch of the direct kernel (M <= 9,
//     no intermediate) or one annihilation + one creation launch through the
//     members' E (hpsi.cu, k_batch_*), blocks assigned from (member, block)
//     work tables;
//   * vector stages: blocks assigned from (member, 2048-row tile) work tables,
//     per-member partial sums reduced in a fixed order by one block per member;
//   * a member whose Lanczos broke down sets its flag and every later block of
//     that member returns at entry (per-member masking);
//   * the lowest eigenvalue of each member's tridiagonal is found on the
//     device by Sturm-sequence bisection (Barth, Martin & Wilkinson 1967), so
//     the whole solve -- start vectors, 120 steps, eigenvalues -- is captured
//     once and replayed with a single cudaGraphLaunch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.h"
#include "space.h"

namespace mcpi {

struct BatchLz {
    int64_t nc;
    double2 *V;        // lm * nc Krylov basis
    double2 *r;        // nc residual (H.psi output)
    double2 *alpha;    // lm
    double *beta;      // lm
    double *maxbeta;   // 1
    int *done;         // 1
    int *iters;        // 1
    double2 *coef;     // lm
    double2 *part;     // (lm + 1) * ceil(nc / kTileMin) partial sums (room for the smallest tile)
    int ntiles;        // ceil(nc / tile) for the batch's tile
};

namespace {

constexpr int kThreads = 256;
// rows per work tile of the vector stages: the autotuner picks one of these
constexpr int kTileCands[3] = {512, 1024, 2048};
constexpr int kTileMin = 512;
constexpr int kUpdBatch = 8;   // basis entries in flight per thread in kb_update

__device__ __forceinline__ double2 warp_sum2(double2 v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// fixed-order block sum, result in thread 0
__device__ __forceinline__ double2 block_sum2(double2 v)
{
    __shared__ double2 red[kThreads / 32];
    v = warp_sum2(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = v;
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (threadIdx.x == 0)
        for (int k = 0; k < kThreads / 32; ++k) {
            r.x += red[k].x;
            r.y += red[k].y;
        }
    return r;
}

__device__ __forceinline__ double2 cmulc(double2 a, double2 b)  // conj(a) b
{
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

__global__ void kb_reset(BatchLz *L, int nmem, int lm)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmem) return;
    *L[m].maxbeta = 0.0;
    *L[m].done = 0;
    *L[m].iters = lm;
}

// partial of <V_a, r> over one tile; with beta_i set, r -= beta_i V_prev first
template <int T>
__global__ void kb_axpy_dot(BatchLz *L, const int2 *__restrict__ work, int i)
{
    const int2 w = work[blockIdx.x];
    BatchLz &b = L[w.x];
    if (*b.done) return;
    const int64_t r0 = (int64_t)w.y * T;
    const int64_t r1 = min(b.nc, r0 + T);
    const double2 *va = b.V + (size_t)(i + 1) * b.nc;
    const double2 *vp = i >= 0 ? b.V + (size_t)i * b.nc : nullptr;
    const double bi = i >= 0 ? b.beta[i] : 0.0;
    double2 acc = make_double2(0.0, 0.0);
    for (int64_t x = r0 + threadIdx.x; x < r1; x += kThreads) {
        double2 y = b.r[x];
        if (vp) {
            const double2 p = vp[x];
            y.x -= bi * p.x;
            y.y -= bi * p.y;
            b.r[x] = y;
        }
        const double2 d = cmulc(va[x], y);
        acc.x += d.x;
        acc.y += d.y;
    }
    acc = block_sum2(acc);
    if (threadIdx.x == 0) b.part[w.y] = acc;
}

// alpha[k] = sum of the member's tile partials (one block per member)
__global__ void kb_sum_alpha(BatchLz *L, int k)
{
    BatchLz &b = L[blockIdx.x];
    if (*b.done) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < b.ntiles; t += kThreads) {
        acc.x += b.part[t].x;
        acc.y += b.part[t].y;
    }
    acc = block_sum2(acc);
    if (threadIdx.x == 0) b.alpha[k] = acc;
}

// part[j * ntiles + tile] = <V_j, r - alpha_cur V_cur> over the tile, j < nvec
template <int T>
__global__ void __launch_bounds__(kThreads) kb_multidot(BatchLz *L, const int2 *__restrict__ work,
                                                        int cur, int nvec)
{
    __shared__ double2 xs[T];
    const int2 w = work[blockIdx.x];
    BatchLz &b = L[w.x];
    if (*b.done) return;
    const int64_t r0 = (int64_t)w.y * T;
    const int rows = (int)min((int64_t)T, b.nc - r0);
    const double2 a = b.alpha[cur];
    const double2 *vc = b.V + (size_t)cur * b.nc + r0;
    for (int t = threadIdx.x; t < rows; t += kThreads) {
        const double2 y = b.r[r0 + t], v = vc[t];
        xs[t] = make_double2(y.x - (a.x * v.x - a.y * v.y), y.y - (a.x * v.y + a.y * v.x));
    }
    __syncthreads();
    const int wid = threadIdx.x / 32, lane = threadIdx.x % 32;
    for (int j = wid; j < nvec; j += kThreads / 32) {
        const double2 *vj = b.V + (size_t)j * b.nc + r0;
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll 4
        for (int t = lane; t < rows; t += 32) {
            const double2 p = cmulc(vj[t], xs[t]);
            acc.x += p.x;
            acc.y += p.y;
        }
        acc = warp_sum2(acc);
        if (lane == 0) b.part[(size_t)j * b.ntiles + w.y] = acc;
    }
}

// coef[j] = sum over tiles (block (member, group of 8 j), one warp per j)
__global__ void kb_coef(BatchLz *L, int nvec)
{
    BatchLz &b = L[blockIdx.x];
    if (*b.done) return;
    const int wid = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int j = blockIdx.y * (kThreads / 32) + wid;
    if (j < nvec) {
        double2 acc = make_double2(0.0, 0.0);
        for (int t = lane; t < b.ntiles; t += 32) {
            acc.x += b.part[(size_t)j * b.ntiles + t].x;
            acc.y += b.part[(size_t)j * b.ntiles + t].y;
        }
        acc = warp_sum2(acc);
        if (lane == 0) b.coef[j] = acc;
    }
}

// r = (r - alpha_cur V_cur) - sum_{j<nvec} coef_j V_j ; part[tile] = |r|^2 over the tile
template <int T>
__global__ void __launch_bounds__(kThreads) kb_update(BatchLz *L, const int2 *__restrict__ work,
                                                      int cur, int nvec)
{
    extern __shared__ double2 cs[];
    const int2 w = work[blockIdx.x];
    BatchLz &b = L[w.x];
    if (*b.done) return;
    for (int j = threadIdx.x; j < nvec; j += kThreads) cs[j] = b.coef[j];
    __syncthreads();
    const int64_t r0 = (int64_t)w.y * T;
    const int64_t r1 = min(b.nc, r0 + T);
    const double2 a = b.alpha[cur];
    const double2 *vc = b.V + (size_t)cur * b.nc;
    double acc = 0.0;
    for (int64_t x = r0 + threadIdx.x; x < r1; x += kThreads) {
        const double2 y = b.r[x], v = vc[x];
        double2 u = make_double2(y.x - (a.x * v.x - a.y * v.y), y.y - (a.x * v.y + a.y * v.x));
        // kUpdBatch basis entries loaded together, then subtracted in order j
        int j = 0;
        for (; j + kUpdBatch <= nvec; j += kUpdBatch) {
            double2 p[kUpdBatch];
#pragma unroll
            for (int q = 0; q < kUpdBatch; ++q) p[q] = b.V[(size_t)(j + q) * b.nc + x];
#pragma unroll
            for (int q = 0; q < kUpdBatch; ++q) {
                const double2 c = cs[j + q];
                u.x -= p[q].x * c.x - p[q].y * c.y;
                u.y -= p[q].x * c.y + p[q].y * c.x;
            }
        }
        for (; j < nvec; ++j) {
            const double2 p = b.V[(size_t)j * b.nc + x], c = cs[j];
            u.x -= p.x * c.x - p.y * c.y;
            u.y -= p.x * c.y + p.y * c.x;
        }
        b.r[x] = u;
        acc += u.x * u.x + u.y * u.y;
    }
    const double2 s = block_sum2(make_double2(acc, 0.0));
    if (threadIdx.x == 0) b.part[w.y] = s;
}

// beta_i and the breakdown test of groundStateLieb.c:287-292 (one block per member)
__global__ void kb_beta(BatchLz *L, int i, double tol)
{
    BatchLz &b = L[blockIdx.x];
    if (*b.done) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = threadIdx.x; t < b.ntiles; t += kThreads) acc.x += b.part[t].x;
    acc = block_sum2(acc);
    if (threadIdx.x == 0) {
        const double bi = sqrt(acc.x);
        b.beta[i] = bi;
        if (*b.maxbeta < bi) *b.maxbeta = bi;
        if (!(bi / *b.maxbeta >= tol)) {
            *b.done = 1;
            *b.iters = i;
        }
    }
}

template <int T>
__global__ void kb_scale(BatchLz *L, const int2 *__restrict__ work, int i)
{
    const int2 w = work[blockIdx.x];
    BatchLz &b = L[w.x];
    if (*b.done) return;
    const int64_t r0 = (int64_t)w.y * T;
    const int64_t r1 = min(b.nc, r0 + T);
    const double bi = b.beta[i];
    double2 *vn = b.V + (size_t)(i + 1) * b.nc;
    for (int64_t x = r0 + threadIdx.x; x < r1; x += kThreads) {
        const double2 y = b.r[x];
        vn[x] = make_double2(y.x / bi, y.y / bi);
    }
}

// Number of eigenvalues of the tridiagonal (d, e) below x (Sturm sequence).
__device__ int sturm_count(const double2 *alpha, const double *beta, int n, double x)
{
    int c = 0;
    double q = 1.0;
    for (int k = 0; k < n; ++k) {
        const double e2 = k > 0 ? beta[k - 1] * beta[k - 1] : 0.0;
        q = alpha[k].x - x - (k > 0 ? e2 / q : 0.0);
        if (q == 0.0) q = -1e-300;   // step off an exact pole
        c += q < 0.0;
    }
    return c;
}

// Lowest eigenvalue of each member's tridiagonal by bisection on the Sturm
// count, from Gershgorin bounds to the resolution of double precision.
__global__ void kb_eig(BatchLz *L, int nmem, double *E0, int *iters)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nmem) return;
    BatchLz &b = L[m];
    const int it = *b.iters;
    const int n = it > 0 ? it : 1;
    double lo = 1e300, hi = -1e300;
    for (int k = 0; k < n; ++k) {
        const double rad = (k > 0 ? fabs(b.beta[k - 1]) : 0.0) + (k + 1 < n ? fabs(b.beta[k]) : 0.0);
        lo = fmin(lo, b.alpha[k].x - rad);
        hi = fmax(hi, b.alpha[k].x + rad);
    }
    for (int s = 0; s < 200 && hi - lo > 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300; ++s) {
        const double mid = 0.5 * (lo + hi);
        if (mid <= lo || mid >= hi) break;
        if (sturm_count(b.alpha, b.beta, n, mid) >= 1) hi = mid;
        else lo = mid;
    }
    E0[m] = 0.5 * (lo + hi);
    iters[m] = it;
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace mcpi

using mcpi::BatchLz;
using mcpi::BatchMember;

struct mcpi_batch_s {
    int count = 0, lm = 0, device = 0;
    cudaStream_t stream = nullptr;
    std::vector<mcpi_space> spaces;
    std::vector<BatchLz> lz;
    std::vector<BatchMember> mem;
    std::vector<double2 *> start;
    char *arena = nullptr;
    char *meta = nullptr;   // device copies of lz, mem, work tables, results
    BatchLz *d_lz = nullptr;
    BatchMember *d_mem = nullptr;
    int2 *d_vwork = nullptr;   // room for the smallest tile's work table
    int nvwork = 0;
    int tile = 0;              // rows per vector-stage tile (0: autotune at the first run)
    bool tuned = false;
    float tune_ms[3] = {0.f, 0.f, 0.f};   // probe time of each candidate tile
    struct Group {
        int M;
        int2 *w1, *w2;     // member-major work tables
        int2 *w1i, *w2i;   // the same blocks interleaved across members (round robin)
        int n1, n2;
        size_t sm1, sm2, sm3;
        bool direct;       // the direct H.psi form (M <= kBatchDirectMaxM; the members hold no E)
        int form;          // kBatch* as captured
        // the real-valued direct form: members in launches of up to
        // batch_chunk_members(M), their block values a kernel parameter
        struct Chunk {
            int2 *w, *wi;   // (slot, block) work tables, member-major / interleaved
            int n;
            std::vector<int> members;
            std::vector<unsigned char> vals;   // filled when the solve is captured
        };
        std::vector<Chunk> chunks;
    };
    std::vector<char> mreal;   // member's block values are real
    std::vector<Group> groups;
    // batched H.psi schedule (the autotuner's second dimension): bit 0 = the
    // M groups run as concurrent graph branches (else one after another),
    // bit 1 = interleaved work tables (else member-major); -1 = autotune
    int hsched = -1;
    float hsched_ms[4] = {0.f, 0.f, 0.f, 0.f};
    std::vector<cudaStream_t> side;    // one per group after the first
    cudaEvent_t ev_fork = nullptr;
    std::vector<cudaEvent_t> ev_join;
    double *d_E0 = nullptr;
    int *d_iters = nullptr;
    std::vector<char> ready;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t arena_bytes = 0;
};

namespace {

int bfail(int code, const std::string &msg) { return mcpi::set_error(code, msg.c_str()); }

}  // namespace

extern "C" {

int mcpi_batch_create(int count, const int *N, const int *M, int lm, int device, mcpi_batch *out)
{
    if (!out || !N || !M || count < 1 || lm < 2 || lm > 2048)
        return bfail(MCPI_ERR_ARG, "mcpi_batch_create: bad arguments");
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return bfail(MCPI_ERR_CUDA, "mcpi_batch_create: bad device");
    auto *b = new mcpi_batch_s;
    b->count = count;
    b->lm = lm;
    b->device = device;
    b->spaces.assign(count, nullptr);
    b->ready.assign(count, 0);
    b->mreal.assign(count, 1);
    auto cleanup = [&](int rc, const std::string &msg) {
        mcpi_batch_destroy(b);
        return bfail(rc, msg);
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
        return cleanup(MCPI_ERR_CUDA, "stream creation failed");
    // sizes
    std::vector<size_t> off_V(count), off_r(count), off_E(count), off_S(count), off_st(count);
    size_t tot = 0;
    b->lz.resize(count);
    b->mem.resize(count);
    for (int m = 0; m < count; ++m) {
        if (N[m] < 2 || M[m] < 2 || M[m] > mcpi::kMaxM)
            return cleanup(MCPI_ERR_RANGE, "batched members need N >= 2 and 2 <= M <= 16");
        int rc = mcpi_space_create(N[m], M[m], device, &b->spaces[m]);
        if (rc) return cleanup(rc, std::string("member space: ") + mcpi_last_error());
        const mcpi_space_s *s = b->spaces[m];
        const int64_t nc = s->nc;
        const int ntiles = (int)((nc + mcpi::kTileMin - 1) / mcpi::kTileMin);   // room for any tile
        b->lz[m].nc = nc;
        b->lz[m].ntiles = ntiles;
        off_V[m] = tot;
        tot += mcpi::up256(sizeof(double2) * (size_t)lm * nc);
        off_r[m] = tot;
        tot += mcpi::up256(sizeof(double2) * nc);
        off_E[m] = tot;
        if (M[m] > mcpi::kBatchDirectMaxM)   // the two-kernel form's intermediate
            tot += mcpi::up256(sizeof(double2) * (size_t)s->P * s->nc2);
        off_S[m] = tot;
        tot += mcpi::up256(sizeof(double2) * nc);
        off_st[m] = tot;
        tot += mcpi::up256(sizeof(double2) * (2 * (size_t)lm + (size_t)(lm + 1) * ntiles) +
                           sizeof(double) * (lm + 1) + 2 * sizeof(int));
    }
    if (cudaMalloc(&b->arena, tot) != cudaSuccess)
        return cleanup(MCPI_ERR_NOMEM, "arena allocation failed (" + std::to_string(tot) + " bytes)");
    b->arena_bytes = tot;
    b->start.resize(count);
    for (int m = 0; m < count; ++m) {
        BatchLz &z = b->lz[m];
        const mcpi_space_s *s = b->spaces[m];
        z.V = reinterpret_cast<double2 *>(b->arena + off_V[m]);
        z.r = reinterpret_cast<double2 *>(b->arena + off_r[m]);
        b->start[m] = reinterpret_cast<double2 *>(b->arena + off_S[m]);
        char *st = b->arena + off_st[m];
        z.alpha = reinterpret_cast<double2 *>(st);
        z.coef = z.alpha + lm;
        z.part = z.coef + lm;
        z.beta = reinterpret_cast<double *>(z.part + (size_t)(lm + 1) * z.ntiles);   // ntiles for kTileMin here
        z.maxbeta = z.beta + lm;
        z.done = reinterpret_cast<int *>(z.maxbeta + 1);
        z.iters = z.done + 1;
        BatchMember &bm = b->mem[m];
        bm.sp = s->sp;
        bm.W = s->d_W;
        bm.sq = s->d_sq;
        bm.hblk = nullptr;
        bm.nh = 0;
        bm.hdiag = nullptr;
        bm.lvec = z.V;
        bm.E = M[m] > mcpi::kBatchDirectMaxM ? reinterpret_cast<double2 *>(b->arena + off_E[m]) : nullptr;
        bm.r = z.r;
        bm.done = z.done;
        bm.occ = bm.occ2 = nullptr;
        bm.occ_bits = 0;
    }
    // work tables: vector tiles of every member, H.psi blocks grouped by M
    std::vector<int2> vwork;
    for (int m = 0; m < count; ++m)
        for (int t = 0; t < b->lz[m].ntiles; ++t) vwork.push_back(make_int2(m, t));
    std::vector<int> Ms(M, M + count);
    std::sort(Ms.begin(), Ms.end());
    Ms.erase(std::unique(Ms.begin(), Ms.end()), Ms.end());
    std::vector<std::vector<int2>> w1(Ms.size()), w2(Ms.size()), w1i(Ms.size()), w2i(Ms.size());
    const int rpb1 = mcpi::batch_rows_per_block(1), rpb2 = mcpi::batch_rows_per_block(2);
    for (size_t g = 0; g < Ms.size(); ++g) {
        int64_t most1 = 0, most2 = 0;
        for (int m = 0; m < count; ++m) {
            if (M[m] != Ms[g]) continue;
            const mcpi_space_s *s = b->spaces[m];
            const int64_t b1 = (s->nc2 + rpb1 - 1) / rpb1, b2 = (s->nc + rpb2 - 1) / rpb2;
            for (int64_t k = 0; k < b1; ++k) w1[g].push_back(make_int2(m, (int)k));
            for (int64_t k = 0; k < b2; ++k) w2[g].push_back(make_int2(m, (int)k));
            most1 = std::max(most1, b1);
            most2 = std::max(most2, b2);
        }
        for (int64_t k = 0; k < most1; ++k)
            for (int m = 0; m < count; ++m)
                if (M[m] == Ms[g] && k < (b->spaces[m]->nc2 + rpb1 - 1) / rpb1) w1i[g].push_back(make_int2(m, (int)k));
        for (int64_t k = 0; k < most2; ++k)
            for (int m = 0; m < count; ++m)
                if (M[m] == Ms[g] && k < (b->spaces[m]->nc + rpb2 - 1) / rpb2) w2i[g].push_back(make_int2(m, (int)k));
    }
    // chunks of the direct groups: (slot, block) tables
    std::vector<std::vector<std::vector<int>>> cmem(Ms.size());
    std::vector<std::vector<std::vector<int2>>> cw(Ms.size()), cwi(Ms.size());
    for (size_t g = 0; g < Ms.size(); ++g) {
        if (Ms[g] > mcpi::kBatchDirectMaxM) continue;
        const int cap = mcpi::batch_chunk_members(Ms[g]);
        for (int m = 0; m < count; ++m) {
            if (M[m] != Ms[g]) continue;
            if (cmem[g].empty() || (int)cmem[g].back().size() == cap) cmem[g].emplace_back();
            cmem[g].back().push_back(m);
        }
        for (const auto &mm : cmem[g]) {
            std::vector<int2> a, ai;
            int64_t most = 0;
            for (size_t sl = 0; sl < mm.size(); ++sl) {
                const int64_t nb = (b->spaces[mm[sl]]->nc + rpb2 - 1) / rpb2;
                for (int64_t k = 0; k < nb; ++k) a.push_back(make_int2((int)sl, (int)k));
                most = std::max(most, nb);
            }
            for (int64_t k = 0; k < most; ++k)
                for (size_t sl = 0; sl < mm.size(); ++sl)
                    if (k < (b->spaces[mm[sl]]->nc + rpb2 - 1) / rpb2) ai.push_back(make_int2((int)sl, (int)k));
            cw[g].push_back(a);
            cwi[g].push_back(ai);
        }
    }
    size_t mbytes = mcpi::up256(sizeof(BatchLz) * count) + mcpi::up256(sizeof(BatchMember) * count) +
                    mcpi::up256(sizeof(int2) * vwork.size()) + mcpi::up256(sizeof(double) * count) +
                    mcpi::up256(sizeof(int) * count);
    for (size_t g = 0; g < Ms.size(); ++g) {
        mbytes += 2 * (mcpi::up256(sizeof(int2) * w1[g].size()) + mcpi::up256(sizeof(int2) * w2[g].size()));
        for (size_t c = 0; c < cw[g].size(); ++c)
            mbytes += mcpi::up256(sizeof(int2) * cw[g][c].size()) + mcpi::up256(sizeof(int2) * cwi[g][c].size());
    }
    if (cudaMalloc(&b->meta, mbytes) != cudaSuccess) return cleanup(MCPI_ERR_NOMEM, "metadata allocation failed");
    char *p = b->meta;
    auto take = [&](size_t bytes) {
        char *q = p;
        p += mcpi::up256(bytes);
        return q;
    };
    b->d_lz = reinterpret_cast<BatchLz *>(take(sizeof(BatchLz) * count));
    b->d_mem = reinterpret_cast<BatchMember *>(take(sizeof(BatchMember) * count));
    b->d_vwork = reinterpret_cast<int2 *>(take(sizeof(int2) * vwork.size()));
    b->nvwork = (int)vwork.size();
    b->d_E0 = reinterpret_cast<double *>(take(sizeof(double) * count));
    b->d_iters = reinterpret_cast<int *>(take(sizeof(int) * count));
    cudaError_t e = cudaMemcpy(b->d_lz, b->lz.data(), sizeof(BatchLz) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_vwork, vwork.data(), sizeof(int2) * vwork.size(), cudaMemcpyHostToDevice);
    for (size_t g = 0; g < Ms.size() && e == cudaSuccess; ++g) {
        mcpi_batch_s::Group G{};
        G.M = Ms[g];
        G.w1 = reinterpret_cast<int2 *>(take(sizeof(int2) * w1[g].size()));
        G.w2 = reinterpret_cast<int2 *>(take(sizeof(int2) * w2[g].size()));
        G.w1i = reinterpret_cast<int2 *>(take(sizeof(int2) * w1i[g].size()));
        G.w2i = reinterpret_cast<int2 *>(take(sizeof(int2) * w2i[g].size()));
        G.n1 = (int)w1[g].size();
        G.n2 = (int)w2[g].size();
        int maxN = 0;
        for (int m = 0; m < count; ++m)
            if (M[m] == Ms[g]) maxN = std::max(maxN, N[m]);
        const int P = Ms[g] * (Ms[g] + 1) / 2;
        int nh = 0;   // momentum-block values: sum over K of (block size)^2
        for (int K = 0; K <= 2 * Ms[g] - 2; ++K) {
            const int qlo = std::max(0, K - (Ms[g] - 1)), n = K / 2 - qlo + 1;
            nh += n * n;
        }
        (void)P;
        G.sm1 = mcpi::batch_smem(Ms[g], maxN, nh, 1);
        G.sm2 = mcpi::batch_smem(Ms[g], maxN, nh, 2);
        G.sm3 = mcpi::batch_smem(Ms[g], maxN, nh, 3);
        G.direct = Ms[g] <= mcpi::kBatchDirectMaxM;
        G.form = mcpi::kBatchTwo;
        e = mcpi::batch_prepare(Ms[g], G.sm1, G.sm2, G.sm3);
        if (e != cudaSuccess) break;
        e = cudaMemcpy(G.w1, w1[g].data(), sizeof(int2) * w1[g].size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G.w2, w2[g].data(), sizeof(int2) * w2[g].size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G.w1i, w1i[g].data(), sizeof(int2) * w1i[g].size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(G.w2i, w2i[g].data(), sizeof(int2) * w2i[g].size(), cudaMemcpyHostToDevice);
        for (size_t c = 0; c < cw[g].size() && e == cudaSuccess; ++c) {
            mcpi_batch_s::Group::Chunk C;
            C.w = reinterpret_cast<int2 *>(take(sizeof(int2) * cw[g][c].size()));
            C.wi = reinterpret_cast<int2 *>(take(sizeof(int2) * cwi[g][c].size()));
            C.n = (int)cw[g][c].size();
            C.members = cmem[g][c];
            C.vals.assign(mcpi::batch_vals_bytes(Ms[g]), 0);
            e = cudaMemcpy(C.w, cw[g][c].data(), sizeof(int2) * cw[g][c].size(), cudaMemcpyHostToDevice);
            if (e == cudaSuccess)
                e = cudaMemcpy(C.wi, cwi[g][c].data(), sizeof(int2) * cwi[g][c].size(), cudaMemcpyHostToDevice);
            G.chunks.push_back(std::move(C));
        }
        b->groups.push_back(G);
    }
    // side streams and events for the concurrent H.psi schedule
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming);
    for (size_t g = 1; g < b->groups.size() && e == cudaSuccess; ++g) {
        cudaStream_t x = nullptr;
        cudaEvent_t y = nullptr;
        e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
        if (e == cudaSuccess) b->side.push_back(x);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&y, cudaEventDisableTiming);
        if (e == cudaSuccess) b->ev_join.push_back(y);
    }
    if (e != cudaSuccess) return cleanup(MCPI_ERR_CUDA, std::string("upload: ") + cudaGetErrorString(e));
    *out = b;
    return MCPI_OK;
}

int mcpi_batch_member_size(mcpi_batch b, int member, int64_t *nc)
{
    if (!b || member < 0 || member >= b->count || !nc) return bfail(MCPI_ERR_ARG, "bad arguments");
    *nc = b->lz[member].nc;
    return MCPI_OK;
}

int mcpi_batch_set_integrals(mcpi_batch b, int member, const double *h_Ho, const double *h_Hint, int variant)
{
    if (!b || member < 0 || member >= b->count) return bfail(MCPI_ERR_ARG, "bad member");
    int rc = mcpi_set_integrals(b->spaces[member], h_Ho, h_Hint, variant);
    if (rc) return bfail(rc, mcpi_last_error());
    const mcpi_space_s *s = b->spaces[member];
    if (!s->fwd.hblk)
        return bfail(MCPI_ERR_ARG, "batched solves need integrals that conserve the total orbital index "
                                   "(momentum-conserving plane-wave integrals)");
    bool real = true;
    for (const double2 &h : s->fwd.hblk_h) real = real && h.y == 0.0;
    b->mreal[member] = real;
    if (b->exec)   // the real-valued direct form carries the values in the graph: capture again
        for (const auto &G : b->groups)
            if (G.M == s->M && G.form == mcpi::kBatchDirectReal && b->exec) {
                cudaStreamSynchronize(b->stream);
                cudaGraphExecDestroy(b->exec);
                cudaGraphDestroy(b->graph);
                b->exec = nullptr;
                b->graph = nullptr;
            }
    BatchMember &bm = b->mem[member];
    bm.hblk = s->fwd.hblk;
    bm.nh = s->fwd.nhblk;
    bm.hdiag = s->fwd.hdiag;
    bm.occ = s->d_occ;
    bm.occ2 = s->d_occ2;
    bm.occ_bits = s->occ_bits;
    b->ready[member] |= 1;
    if (cudaMemcpy(b->d_mem + member, &bm, sizeof(BatchMember), cudaMemcpyHostToDevice) != cudaSuccess)
        return bfail(MCPI_ERR_CUDA, "member upload failed");
    return MCPI_OK;
}

int mcpi_batch_set_start(mcpi_batch b, int member, const void *C)
{
    if (!b || member < 0 || member >= b->count || !C) return bfail(MCPI_ERR_ARG, "bad arguments");
    if (cudaSetDevice(b->device) != cudaSuccess ||
        cudaMemcpy(b->start[member], C, sizeof(double2) * b->lz[member].nc, cudaMemcpyDefault) != cudaSuccess)
        return bfail(MCPI_ERR_CUDA, "start vector copy failed");
    b->ready[member] |= 2;
    return MCPI_OK;
}

}  // extern "C"

// Rows per vector-stage tile: per-member tile counts and the (member, tile)
// work table of every vector stage follow it.
static cudaError_t set_tile(mcpi_batch b, int T)
{
    std::vector<int2> vwork;
    for (int m = 0; m < b->count; ++m) {
        b->lz[m].ntiles = (int)((b->lz[m].nc + T - 1) / T);
        for (int t = 0; t < b->lz[m].ntiles; ++t) vwork.push_back(make_int2(m, t));
    }
    cudaError_t e = cudaMemcpy(b->d_lz, b->lz.data(), sizeof(BatchLz) * b->count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_vwork, vwork.data(), sizeof(int2) * vwork.size(), cudaMemcpyHostToDevice);
    b->nvwork = (int)vwork.size();
    b->tile = T;
    return e;
}

// One batched H.psi of Krylov vector vec under H.psi schedule sched (bits as
// mcpi_batch_s::hsched): the M groups one after another on the batch's
// stream, or as concurrent branches (side streams forked from and joined back
// into it -- graph branches under capture).
static cudaError_t enqueue_hpsi(mcpi_batch b, int vec, int sched)
{
    cudaStream_t st = b->stream;
    const bool branches = (sched & 1) && b->groups.size() > 1, inter = (sched & 2) != 0;
    cudaError_t e = cudaSuccess;
    if (branches) {
        e = cudaEventRecord(b->ev_fork, st);
        for (size_t g = 1; g < b->groups.size() && e == cudaSuccess; ++g)
            e = cudaStreamWaitEvent(b->side[g - 1], b->ev_fork, 0);
    }
    for (size_t g = 0; g < b->groups.size() && e == cudaSuccess; ++g) {
        const auto &G = b->groups[g];
        cudaStream_t s = branches && g > 0 ? b->side[g - 1] : st;
        if (G.form == mcpi::kBatchDirectReal)
            for (size_t c = 0; c < G.chunks.size() && e == cudaSuccess; ++c)
                e = mcpi::launch_batch_direct_vals(G.M, b->d_mem, inter ? G.chunks[c].wi : G.chunks[c].w,
                                                   G.chunks[c].n, G.sm3, vec, G.chunks[c].vals.data(), s);
        else
            e = mcpi::launch_batch_apply_h(G.M, G.form, b->d_mem, inter ? G.w1i : G.w1, G.n1, G.sm1,
                                           inter ? G.w2i : G.w2, G.n2, G.direct ? G.sm3 : G.sm2, vec, s);
        if (e == cudaSuccess && branches && g > 0) e = cudaEventRecord(b->ev_join[g - 1], s);
    }
    if (branches)
        for (size_t g = 1; g < b->groups.size() && e == cudaSuccess; ++g)
            e = cudaStreamWaitEvent(st, b->ev_join[g - 1], 0);
    return e;
}

template <int T>
static cudaError_t enqueue_solve_t(mcpi_batch b)
{
    cudaStream_t st = b->stream;
    const int lm = b->lm, nm = b->count;
    cudaError_t e = cudaSuccess;
    for (int m = 0; m < nm && e == cudaSuccess; ++m)
        e = cudaMemcpyAsync(b->lz[m].V, b->start[m], sizeof(double2) * b->lz[m].nc, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    mcpi::kb_reset<<<(nm + 127) / 128, 128, 0, st>>>(b->d_lz, nm, lm);
    auto hpsi = [&](int vec) { return enqueue_hpsi(b, vec, b->hsched); };
    const int nw = b->nvwork;
    e = hpsi(0);
    if (e != cudaSuccess) return e;
    mcpi::kb_axpy_dot<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, -1);
    mcpi::kb_sum_alpha<<<nm, mcpi::kThreads, 0, st>>>(b->d_lz, 0);
    mcpi::kb_update<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, 0, 0);
    for (int i = 0; i < lm - 1; ++i) {
        mcpi::kb_beta<<<nm, mcpi::kThreads, 0, st>>>(b->d_lz, i, 1e-15);
        mcpi::kb_scale<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, i);
        e = hpsi(i + 1);
        if (e != cudaSuccess) return e;
        mcpi::kb_axpy_dot<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, i);
        mcpi::kb_sum_alpha<<<nm, mcpi::kThreads, 0, st>>>(b->d_lz, i + 1);
        mcpi::kb_multidot<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, i + 1, i + 2);
        mcpi::kb_coef<<<dim3(nm, (i + 2 + 7) / 8), mcpi::kThreads, 0, st>>>(b->d_lz, i + 2);
        mcpi::kb_update<T><<<nw, mcpi::kThreads, sizeof(double2) * (i + 2), st>>>(b->d_lz, b->d_vwork, i + 1,
                                                                                    i + 2);
    }
    mcpi::kb_eig<<<(nm + 127) / 128, 128, 0, st>>>(b->d_lz, nm, b->d_E0, b->d_iters);
    return cudaGetLastError();
}

static cudaError_t enqueue_solve(mcpi_batch b)
{
    switch (b->tile) {
    case 512: return enqueue_solve_t<512>(b);
    case 1024: return enqueue_solve_t<1024>(b);
    case 2048: return enqueue_solve_t<2048>(b);
    default: return cudaErrorInvalidValue;
    }
}

// One Lanczos step's vector stages at half the basis size (r -= beta v with the
// alpha dot, the two reorthogonalisation passes, the scaling), on this batch's
// own arena; the solve that follows re-initialises everything they touch.
template <int T>
static cudaError_t probe_tile(mcpi_batch b, int nvec)
{
    cudaStream_t st = b->stream;
    const int nw = b->nvwork;
    mcpi::kb_axpy_dot<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, nvec - 2);
    mcpi::kb_multidot<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, nvec - 1, nvec);
    mcpi::kb_update<T><<<nw, mcpi::kThreads, sizeof(double2) * nvec, st>>>(b->d_lz, b->d_vwork, nvec - 1, nvec);
    mcpi::kb_scale<T><<<nw, mcpi::kThreads, 0, st>>>(b->d_lz, b->d_vwork, nvec - 2);
    return cudaGetLastError();
}

// The autotuner: times the vector stages with each candidate tile (CUDA
// events, best of three after a warm-up) and keeps the fastest.
static cudaError_t autotune(mcpi_batch b)
{
    const int nvec = b->lm / 2 > 2 ? b->lm / 2 : 2;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    int best = -1;
    for (int c = 0; c < 3 && e == cudaSuccess; ++c) {
        const int T = mcpi::kTileCands[c];
        e = set_tile(b, T);
        if (e != cudaSuccess) break;
        mcpi::kb_reset<<<(b->count + 127) / 128, 128, 0, b->stream>>>(b->d_lz, b->count, b->lm);
        float ms = 1e30f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(e0, b->stream);
            if (e == cudaSuccess)
                e = T == 512 ? probe_tile<512>(b, nvec) : T == 1024 ? probe_tile<1024>(b, nvec) : probe_tile<2048>(b, nvec);
            if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float t = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0 && t < ms) ms = t;   // the first repetition warms up
        }
        b->tune_ms[c] = ms;
        if (best < 0 || ms < b->tune_ms[best]) best = c;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e == cudaSuccess) e = set_tile(b, mcpi::kTileCands[best]);
    b->tuned = e == cudaSuccess;
    return e;
}

// The autotuner's H.psi dimension: one batched H.psi of the start vectors
// under each schedule (CUDA events, best of three after a warm-up); keeps the
// fastest. The schedule does not change any member's arithmetic.
static cudaError_t autotune_hpsi(mcpi_batch b)
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    for (int m = 0; m < b->count && e == cudaSuccess; ++m)
        e = cudaMemcpyAsync(b->lz[m].V, b->start[m], sizeof(double2) * b->lz[m].nc, cudaMemcpyDeviceToDevice,
                            b->stream);
    if (e == cudaSuccess) mcpi::kb_reset<<<(b->count + 127) / 128, 128, 0, b->stream>>>(b->d_lz, b->count, b->lm);
    int best = -1;
    for (int c = 0; c < 4 && e == cudaSuccess; ++c) {
        float ms = 1e30f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(e0, b->stream);
            if (e == cudaSuccess) e = enqueue_hpsi(b, 0, c);
            if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float t = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
            if (rep > 0 && t < ms) ms = t;
        }
        b->hsched_ms[c] = ms;
        if (best < 0 || ms < b->hsched_ms[best]) best = c;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (e == cudaSuccess) b->hsched = best;
    return e;
}

extern "C" {

int mcpi_batch_set_schedule(mcpi_batch b, int tile_rows)
{
    if (!b) return bfail(MCPI_ERR_ARG, "null batch");
    if (b->exec) return bfail(MCPI_ERR_STATE, "mcpi_batch_set_schedule: the solve has already been captured");
    if (tile_rows != 0 && tile_rows != 512 && tile_rows != 1024 && tile_rows != 2048)
        return bfail(MCPI_ERR_ARG, "mcpi_batch_set_schedule: tile_rows must be 0, 512, 1024 or 2048");
    b->tile = tile_rows;
    b->tuned = false;
    return MCPI_OK;
}

int mcpi_batch_set_hpsi_schedule(mcpi_batch b, int schedule)
{
    if (!b) return bfail(MCPI_ERR_ARG, "null batch");
    if (b->exec) return bfail(MCPI_ERR_STATE, "mcpi_batch_set_hpsi_schedule: the solve has already been captured");
    if (schedule < -1 || schedule > 3) return bfail(MCPI_ERR_ARG, "mcpi_batch_set_hpsi_schedule: schedule must be -1 .. 3");
    b->hsched = schedule;
    for (float &x : b->hsched_ms) x = 0.f;
    return MCPI_OK;
}

int mcpi_batch_hpsi_schedule(mcpi_batch b, int *schedule, float *h_ms)
{
    if (!b) return bfail(MCPI_ERR_ARG, "null batch");
    if (schedule) *schedule = b->exec ? b->hsched : -1;
    if (h_ms)
        for (int c = 0; c < 4; ++c) h_ms[c] = b->hsched_ms[c];
    return MCPI_OK;
}

int mcpi_batch_schedule(mcpi_batch b, int *tile_rows, float *h_ms)
{
    if (!b) return bfail(MCPI_ERR_ARG, "null batch");
    if (tile_rows) *tile_rows = b->exec ? b->tile : 0;
    if (h_ms)
        for (int c = 0; c < 3; ++c) h_ms[c] = b->tuned ? b->tune_ms[c] : 0.f;
    return MCPI_OK;
}

int mcpi_batch_run(mcpi_batch b, double *h_E0, int *h_iters)
{
    if (!b) return bfail(MCPI_ERR_ARG, "null batch");
    for (int m = 0; m < b->count; ++m)
        if (b->ready[m] != 3) return bfail(MCPI_ERR_STATE, "every member needs integrals and a start vector");
    if (cudaSetDevice(b->device) != cudaSuccess) return bfail(MCPI_ERR_CUDA, "cudaSetDevice failed");
    cudaError_t e = cudaSuccess;
    if (!b->exec) {
        for (auto &G : b->groups) {   // the H.psi form of each M group, fixed in the graph
            bool real = true;
            for (int m = 0; m < b->count; ++m)
                if (b->spaces[m]->M == G.M) real = real && b->mreal[m];
            G.form = !G.direct ? mcpi::kBatchTwo : real ? mcpi::kBatchDirectReal : mcpi::kBatchDirectComplex;
            if (G.form == mcpi::kBatchDirectReal)
                for (auto &C : G.chunks)
                    for (size_t sl = 0; sl < C.members.size(); ++sl)
                        mcpi::batch_fill_vals(G.M, C.vals.data(), (int)sl, C.members[sl],
                                              b->spaces[C.members[sl]]->fwd.hblk_h.data());
        }
        e = b->tile == 0 ? autotune(b) : set_tile(b, b->tile);
        if (e == cudaSuccess && b->hsched < 0) e = autotune_hpsi(b);
        if (e != cudaSuccess) return bfail(MCPI_ERR_CUDA, std::string("batch schedule: ") + cudaGetErrorString(e));
        e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t q = enqueue_solve(b);
            e = cudaStreamEndCapture(b->stream, &b->graph);
            if (q != cudaSuccess) e = q;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (e != cudaSuccess) return bfail(MCPI_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    e = cudaGraphLaunch(b->exec, b->stream);
    if (e == cudaSuccess && h_E0)
        e = cudaMemcpyAsync(h_E0, b->d_E0, sizeof(double) * b->count, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess && h_iters)
        e = cudaMemcpyAsync(h_iters, b->d_iters, sizeof(int) * b->count, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return bfail(MCPI_ERR_CUDA, std::string("batch run: ") + cudaGetErrorString(e));
    return MCPI_OK;
}

int mcpi_batch_arena_bytes(mcpi_batch b, size_t *bytes)
{
    if (!b || !bytes) return bfail(MCPI_ERR_ARG, "bad arguments");
    *bytes = b->arena_bytes;
    return MCPI_OK;
}

int mcpi_batch_destroy(mcpi_batch b)
{
    if (!b) return MCPI_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (mcpi_space s : b->spaces) mcpi_space_destroy(s);
    cudaFree(b->arena);
    cudaFree(b->meta);
    for (cudaStream_t x : b->side) cudaStreamDestroy(x);
    for (cudaEvent_t x : b->ev_join) cudaEventDestroy(x);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return MCPI_OK;
}

}  // extern "C"

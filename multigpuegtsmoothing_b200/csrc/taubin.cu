// Taubin lambda/mu smoothing over the EGT-filtered CSR neighbourhoods.
//
// Reference: taubin_step_GKNN (EGT_CUDA.cu:229-276) driven by PerformSmoothing
// (EGT_CUDA.cu:559-633): per half-step
//     p' = p + s * sum_j w_j (q_j - p) / sum_j w_j,   w_j = expf(-|p - q_j|^2),
// s = lambda then mu, sum = 1e-8 when no neighbour contributes (isRegularized = 0,
// EGT_CUDA.cu:544).  The reference reads the full n*k list (including the -1
// entries the filter left) with three scalar gathers per neighbour, launches in
// 2M-thread chunks and synchronises after each of the 2*iters launches.
//
// Here: one thread per point walks its CSR row (kept neighbours only, in list
// order, so the floating-point accumulation order and therefore the result are
// identical to the reference's); positions are float4 (one 16-byte gather per
// neighbour); the 2*iters launches are captured once into a CUDA graph cached
// on the handle.  For the loop the working set is relabelled into Morton order
// of the level-0 cells: consecutive points then form compact 3-D blobs, so the
// neighbours of a 256-row tile are few and mostly inside the tile; each
// distinct neighbour position is gathered into shared memory once per tile and
// the rows read them from there.  Inside a tile the rows are then ordered by
// decreasing neighbour count, so that the threads of a warp have equal work.
// Relabelling changes neither a row's neighbour order nor any value, so the
// result is the same bit for bit.  Each half-step is a programmatic dependent
// launch: its prologue (CSR tables only) overlaps the previous half-step.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cub/cub.cuh>
#include "egt_internal.cuh"

namespace egt {
namespace {

constexpr int kBatch = 8;        // neighbour gathers in flight per thread
constexpr int kTile = 256;       // rows per block
constexpr int kTileCap = 4608;   // CSR entries per staged tile (the 4M workload peaks at ~4.5k)

// One neighbour's contribution.  The squared distance is contracted as the
// reference build contracts norm2_GKNN inside taubin_step_GKNN --
// fma(dz,dz, fma(dy,dy, dx*dx)), found by comparing candidate contractions
// against the reference's own smoothed positions (0 mismatches on three
// fixtures).
//
// The reference also forms q - p for the weighted sum.  Round-to-nearest
// subtraction is antisymmetric, so q - p is exactly -(p - q) and the fused
// multiply-adds below take the negated difference instead of a second
// subtraction.  The one case where the two differ in sign bit -- a zero
// difference -- gives w * (+-0) + c == c for every reachable c (the sums start
// at +0 and never become -0), so the result is unchanged bit for bit.
__device__ __forceinline__ void accumulate(float x1, float y1, float z1, float4 q, float& cx, float& cy,
                                           float& cz, float& sum) {
    const float dx = __fsub_rn(x1, q.x), dy = __fsub_rn(y1, q.y), dz = __fsub_rn(z1, q.z);
    const float distance = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    const float w = expf(-distance);
    cx = __fmaf_rn(w, -dx, cx);
    cy = __fmaf_rn(w, -dy, cy);
    cz = __fmaf_rn(w, -dz, cz);
    sum = __fadd_rn(sum, w);
}

__device__ __forceinline__ float4 finish(float4 p, float cx, float cy, float cz, float sum, float scale) {
    if (sum == 0.0f) sum = 1e-8f;
    float4 o;
    o.x = __fadd_rn(p.x, __fdiv_rn(__fmul_rn(scale, cx), sum));
    o.y = __fadd_rn(p.y, __fdiv_rn(__fmul_rn(scale, cy), sum));
    o.z = __fadd_rn(p.z, __fdiv_rn(__fmul_rn(scale, cz), sum));
    o.w = p.w;  // keeps whatever the caller stores there (the packed cell coordinates)
    return o;
}

// Row walk with kBatch independent gathers in flight, accumulation in order.
// Entry e of the row is cols[e - cbase].
__device__ __forceinline__ float4 row_update(const float4* __restrict__ pin, const int* cols, int cbase, int e0,
                                             int e1, int self, float scale) {
    const float4 p = __ldg(pin + self);
    float cx = 0.0f, cy = 0.0f, cz = 0.0f, sum = 0.0f;
    for (int e = e0; e < e1; e += kBatch) {
        const int cnt = min(kBatch, e1 - e);
        int j[kBatch];
        float4 q[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; u++) j[u] = u < cnt ? cols[e + u - cbase] : self;
#pragma unroll
        for (int u = 0; u < kBatch; u++) q[u] = __ldg(pin + j[u]);
#pragma unroll
        for (int u = 0; u < kBatch; u++)
            if (u < cnt) accumulate(p.x, p.y, p.z, q[u], cx, cy, cz, sum);
    }
    return finish(p, cx, cy, cz, sum, scale);
}

// General half-step: any CSR, any point order (used by egt_taubin_noalloc).
__global__ void __launch_bounds__(256) k_taubin(const float4* __restrict__ pin, float4* __restrict__ pout,
                                                const int* __restrict__ off, const int* __restrict__ col, int n,
                                                float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    pout[i] = row_update(pin, col, 0, __ldg(off + i), __ldg(off + i + 1), i, scale);
}

// Programmatic dependent launch (griddepcontrol): wait() blocks until the
// preceding grid in the stream has completed and its writes are visible (it
// returns at once when the kernel was not launched as a dependent);
// launch_dependents() lets the next grid start its prologue on free SMs.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;"); }

constexpr int kUCap = 1024;      // distinct neighbours staged per tile (16 KB; 99.8% of tiles fit)
constexpr int kUPer = kUCap / kTile;  // staged positions per thread
constexpr int kSlices = kTile / 32;   // one 32-row slice per warp
constexpr int kSellWords = 1792; // 32-bit slot words per tile (three 10-bit slots each; every tile of the 4M workload fits)
constexpr size_t kStageBytes = kUCap * sizeof(float4) + kSellWords * sizeof(uint32_t);
constexpr int kStages = 2;       // tile buffers per block: one being computed, one being filled
constexpr size_t kPipeSmem = kStages * kStageBytes;
constexpr int kSoffWords = kSlices + 1;  // per tile: slice offsets and the tile's slot count
static_assert(kSellWords % 4 == 0, "slot tables are copied in 4-word vectors");
static_assert(kUCap <= 1024, "slots are 10-bit");
static_assert(kStageBytes % 16 == 0, "stage buffers stay 16-byte aligned");

// 16-byte global -> shared copies that complete asynchronously (cp.async,
// bypassing L1); commit() closes a group, wait<N>() waits until at most N of
// the calling thread's groups are still in flight.
__device__ __forceinline__ void cp_async16(void* dst_smem, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// What a thread needs to know about one tile before its data arrive: the
// tile's distinct-neighbour count, this thread's share of their point
// indices, its row's CSR range, and its warp's slice offset and the tile's
// slot-table size.  Reads only the tile tables, which no half-step writes.
struct TileRegs {
    int nu, e0, e1, soff, ssize;
    int uni[kUPer];
};

__device__ __forceinline__ TileRegs tile_regs(const int* __restrict__ off, const int* __restrict__ t_uni,
                                              const int* __restrict__ t_nu, const int* __restrict__ t_soff,
                                              int tile, int n) {
    TileRegs r;
    const int i = tile * kTile + (int)threadIdx.x;
    r.nu = __ldg(t_nu + tile);
    r.e0 = i < n ? __ldg(off + i) : 0;
    r.e1 = i < n ? __ldg(off + i + 1) : 0;
    r.soff = r.nu >= 0 ? __ldg(t_soff + (size_t)tile * kSoffWords + (threadIdx.x >> 5)) : 0;
    r.ssize = r.nu >= 0 ? __ldg(t_soff + (size_t)tile * kSoffWords + kSlices) : 0;
#pragma unroll
    for (int u = 0; u < kUPer; u++) {
        const int j = (int)threadIdx.x + u * kTile;
        r.uni[u] = (r.nu >= 0 && j < r.nu) ? __ldg(t_uni + (size_t)tile * kUCap + j) : 0;
    }
    return r;
}

// Starts the copies of one tile into a stage buffer: the tile's packed
// neighbour slots (a fixed-stride, 16-byte aligned table of 32-bit words) and
// its staged positions (one 16-byte gather each).  Always commits one group.
__device__ __forceinline__ void tile_fetch(const TileRegs& r, const float4* __restrict__ pin,
                                           const uint32_t* __restrict__ t_loc, int tile, unsigned char* stage) {
    if (r.nu >= 0) {
        float4* s_pos = reinterpret_cast<float4*>(stage);
        uint32_t* s_loc = reinterpret_cast<uint32_t*>(stage + kUCap * sizeof(float4));
        const uint32_t* src = t_loc + (size_t)tile * kSellWords;
        const int nvec = (r.ssize + 3) >> 2;
        for (int v = (int)threadIdx.x; v < nvec; v += kTile) cp_async16(s_loc + 4 * v, src + 4 * v);
#pragma unroll
        for (int u = 0; u < kUPer; u++) {
            const int j = (int)threadIdx.x + u * kTile;
            if (j < r.nu) cp_async16(s_pos + j, pin + r.uni[u]);
        }
    }
    cp_async_commit();
}

// Staged half-step, persistent and double-buffered.  Every kTile-row tile
// has its staged neighbour positions (t_uni: point index of each position
// slot, precomputed once per CSR) and, per CSR entry, the 16-bit slot of its
// neighbour (t_loc).  Block b takes tiles b, b + gridDim.x, ...; while it
// computes one tile from shared memory, the copies of its next tile are in
// flight into the other buffer, and the registers for the tile after that
// are being loaded.  Each distinct neighbour position is fetched from global
// memory once per tile; each row reads its neighbours from shared memory in
// list order.  Tiles that do not fit (t_nu < 0) gather from global memory.
//
// The slots are 10 bits, three to a 32-bit word, sliced by warp: warp w's 32
// rows (ordered by decreasing neighbour count, see morton_prepare) store
// entries 3g..3g+2 of lane l in word soff[w] + 32 g + l, so each step of a
// warp (three neighbours per lane) reads 128 contiguous bytes of slots.  The
// staged tables are what most of the kernel's DRAM traffic is made of; packed
// this way they take 1.3 bytes per entry.
__global__ void __launch_bounds__(kTile, 4) k_taubin_tiles(const float4* __restrict__ pin, float4* __restrict__ pout,
                                                        const int* __restrict__ off, const int* __restrict__ col,
                                                        const int* __restrict__ t_uni,
                                                        const uint32_t* __restrict__ t_loc,
                                                        const int* __restrict__ t_nu, const int* __restrict__ t_soff,
                                                        int n, int tiles, float scale) {
    extern __shared__ __align__(16) unsigned char smem[];
    int tile = blockIdx.x;
    if (tile >= tiles) return;
    const int lane = threadIdx.x & 31;
    // Before grid_dependency_wait() only the tile tables are read: under
    // programmatic dependent launch this overlaps the previous half-step.
    TileRegs cur = tile_regs(off, t_uni, t_nu, t_soff, tile, n);
    int next = tile + gridDim.x;
    TileRegs nxt = next < tiles ? tile_regs(off, t_uni, t_nu, t_soff, next, n) : cur;
    grid_dependency_wait();  // the previous half-step's positions are complete
    grid_dependents_launch();
    tile_fetch(cur, pin, t_loc, tile, smem);
    int i = tile * kTile + (int)threadIdx.x;
    float4 p = i < n ? __ldg(pin + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = 0; tile < tiles; j++) {
        unsigned char* stage = smem + (j & 1) * kStageBytes;
        cp_async_wait<0>();  // this thread's copies of the current tile have landed
        // One barrier per tile: past it, every thread's copies of the current
        // tile are visible, and every thread has finished the previous tile,
        // so the other buffer is free for the next tile's copies.
        __syncthreads();
        float4 p_next = p;
        if (next < tiles) {
            tile_fetch(nxt, pin, t_loc, next, smem + ((j + 1) & 1) * kStageBytes);
            const int in = next * kTile + (int)threadIdx.x;
            if (in < n) p_next = __ldg(pin + in);
        }
        const int after = next + (int)gridDim.x;
        const TileRegs nn = after < tiles ? tile_regs(off, t_uni, t_nu, t_soff, after, n) : nxt;
        if (i < n) {
            float cx = 0.0f, cy = 0.0f, cz = 0.0f, sum = 0.0f;
            if (cur.nu < 0) {  // tile too large to stage: plain gathers
                for (int e = cur.e0; e < cur.e1; e++)
                    accumulate(p.x, p.y, p.z, __ldg(pin + __ldg(col + e)), cx, cy, cz, sum);
            } else {
                const float4* s_pos = reinterpret_cast<const float4*>(stage);
                const uint32_t* ls =
                    reinterpret_cast<const uint32_t*>(stage + kUCap * sizeof(float4)) + cur.soff + lane;
                const int len = cur.e1 - cur.e0;
                // three neighbours per step; the next step's slot word is loaded
                // before this step's positions are read, off the critical path
                int e = 0;
                uint32_t v = len > 0 ? ls[0] : 0u;
#pragma unroll 1
                for (; e + 3 <= len; e += 3) {
                    ls += 32;
                    const uint32_t vn = e + 3 < len ? *ls : v;
                    const float4 q0 = s_pos[v & 1023u], q1 = s_pos[(v >> 10) & 1023u], q2 = s_pos[v >> 20];
                    accumulate(p.x, p.y, p.z, q0, cx, cy, cz, sum);
                    accumulate(p.x, p.y, p.z, q1, cx, cy, cz, sum);
                    accumulate(p.x, p.y, p.z, q2, cx, cy, cz, sum);
                    v = vn;
                }
                if (e < len) {
                    accumulate(p.x, p.y, p.z, s_pos[v & 1023u], cx, cy, cz, sum);
                    if (e + 1 < len) accumulate(p.x, p.y, p.z, s_pos[(v >> 10) & 1023u], cx, cy, cz, sum);
                }
            }
            pout[i] = finish(p, cx, cy, cz, sum, scale);
        }
        tile = next;
        next = after;
        cur = nxt;
        nxt = nn;
        p = p_next;
        i = tile * kTile + (int)threadIdx.x;
    }
    cp_async_wait<0>();
}

// Builds the tables of one tile (one block per tile): a block radix sort of
// the tile's column indices and a unique pass give the distinct neighbours
// (t_uni, at a fixed stride of kUCap per tile) and each CSR entry's index
// into them, a 10-bit slot; the slots are stored three to a 32-bit word,
// sliced by warp (warp w's 32 rows padded to its longest row rounded up to 3,
// entry 3g + j of lane l in bits 10j..10j+9 of word soff[w] + 32 g + l;
// t_soff = soff[0..8] in words, soff[8] the table size).  t_nu = the distinct
// count, or -1 when the tile does not fit (too many entries, distinct
// neighbours or slot words): its rows then gather from global memory, and the
// tile is counted in *spilled.
constexpr int kBuildThreads = 512;
constexpr int kBuildItems = kTileCap / kBuildThreads;

__global__ void __launch_bounds__(kBuildThreads) k_tile_build(const int* __restrict__ off, const int* __restrict__ col,
                                                              int n, int* __restrict__ t_uni,
                                                              uint32_t* __restrict__ t_loc, int* __restrict__ t_nu,
                                                              int* __restrict__ t_soff,
                                                              unsigned long long* __restrict__ spilled) {
    using Sort = cub::BlockRadixSort<int, kBuildThreads, kBuildItems>;
    using Scan = cub::BlockScan<int, kBuildThreads>;
    __shared__ union {
        typename Sort::TempStorage sort;
        int uniq[kTileCap];
    } sm;
    __shared__ typename Scan::TempStorage scan;
    __shared__ int s_last[kBuildThreads];
    __shared__ uint16_t s_u[kTileCap];  // entry -> distinct index
    __shared__ int s_len[kTile], s_start[kTile];
    __shared__ int s_soff[kSoffWords];
    __shared__ int s_nu;
    const int tile = blockIdx.x;
    const int base = tile * kTile;
    const int last = min(base + kTile, n);
    const int rows = last - base;
    const int e_lo = off[base], e_hi = off[last];
    const int cnt = e_hi - e_lo;
    if (cnt > kTileCap) {
        if (threadIdx.x == 0) { t_nu[tile] = -1; atomicAdd(spilled, 1ull); }
        return;
    }
    int keys[kBuildItems];
#pragma unroll
    for (int j = 0; j < kBuildItems; j++) {
        const int i = threadIdx.x * kBuildItems + j;
        keys[j] = i < cnt ? col[e_lo + i] : INT_MAX;
    }
    Sort(sm.sort).Sort(keys);
    s_last[threadIdx.x] = keys[kBuildItems - 1];
    __syncthreads();
    int prev = threadIdx.x > 0 ? s_last[threadIdx.x - 1] : -1;
    int first[kBuildItems];
    int mine = 0;
#pragma unroll
    for (int j = 0; j < kBuildItems; j++) {
        first[j] = keys[j] != INT_MAX && keys[j] != prev;
        mine += first[j];
        prev = keys[j];
    }
    int at = 0, total = 0;
    Scan(scan).ExclusiveSum(mine, at, total);
    __syncthreads();  // the sort storage is reused for the unique list
#pragma unroll
    for (int j = 0; j < kBuildItems; j++)
        if (first[j]) sm.uniq[at++] = keys[j];
    if (threadIdx.x == 0) s_nu = total;
    for (int r = threadIdx.x; r < kTile; r += kBuildThreads) {
        s_len[r] = r < rows ? off[base + r + 1] - off[base + r] : 0;
        s_start[r] = r < rows ? off[base + r] - e_lo : 0;
    }
    __syncthreads();
    const int nu = s_nu;
    if (nu > kUCap) {
        if (threadIdx.x == 0) { t_nu[tile] = -1; atomicAdd(spilled, 1ull); }
        return;
    }
    for (int i = threadIdx.x; i < cnt; i += kBuildThreads) {
        const int v = col[e_lo + i];
        int lo = 0, hi = nu - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (sm.uniq[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        s_u[i] = (uint16_t)lo;
    }
    if (threadIdx.x == 0) {
        s_soff[0] = 0;
        for (int w = 0; w < kSlices; w++) {
            int wmax = 0;
            for (int l = 0; l < 32; l++) wmax = max(wmax, s_len[32 * w + l]);
            s_soff[w + 1] = s_soff[w] + 32 * ((wmax + 2) / 3);
        }
    }
    __syncthreads();
    if (s_soff[kSlices] > kSellWords) {
        if (threadIdx.x == 0) { t_nu[tile] = -1; atomicAdd(spilled, 1ull); }
        return;
    }
    for (int u = threadIdx.x; u < nu; u += kBuildThreads) t_uni[(size_t)tile * kUCap + u] = sm.uniq[u];
    const int ssize = s_soff[kSlices];
    for (int x = threadIdx.x; x < ssize; x += kBuildThreads) {
        int w = 0;
        while (x >= s_soff[w + 1]) w++;
        const int rel = x - s_soff[w], g = rel >> 5, r = 32 * w + (rel & 31);
        uint32_t word = 0;
        for (int j = 0; j < 3; j++) {
            const int e = 3 * g + j;
            if (e < s_len[r]) word |= (uint32_t)s_u[s_start[r] + e] << (10 * j);
        }
        t_loc[(size_t)tile * kSellWords + x] = word;
    }
    if (threadIdx.x < kSoffWords) t_soff[(size_t)tile * kSoffWords + threadIdx.x] = s_soff[threadIdx.x];
    if (threadIdx.x == 0) t_nu[tile] = nu;
}

__global__ void k_split_soa(const float4* __restrict__ p4, int n, float* __restrict__ x, float* __restrict__ y,
                            float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = p4[i];
    x[i] = v.x; y[i] = v.y; z[i] = v.z;
}

// 30-bit Morton code of a packed level-0 cell (x | y<<10 | z<<20).
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__global__ void k_morton_keys(const uint32_t* __restrict__ cell0, int n, uint32_t* __restrict__ key,
                              int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t c = cell0[s];
    key[s] = spread3(c) | (spread3(c >> 10) << 1) | (spread3(c >> 20) << 2);
    idx[s] = s;
}

// Batched clouds: the cloud id above the Morton key keeps each cloud's rows together.
__global__ void k_morton_keys64(const uint32_t* __restrict__ cell0, const uint16_t* __restrict__ cloud, int n,
                                unsigned long long* __restrict__ key, int* __restrict__ idx) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t c = cell0[s];
    key[s] = ((unsigned long long)cloud[s] << 30) | (spread3(c) | (spread3(c >> 10) << 1) | (spread3(c >> 20) << 2));
    idx[s] = s;
}

// Sort keys that order the rows of every kTile-row tile of the Morton order
// by decreasing neighbour count; a stable sort keeps equal counts in Morton
// order.
__global__ void k_degree_keys(const int* __restrict__ perm, const int* __restrict__ off, int n,
                              uint32_t* __restrict__ key, int* __restrict__ val) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = perm[i];
    const int len = min(off[s + 1] - off[s], 255);
    key[i] = ((uint32_t)(i / kTile) << 8) | (uint32_t)(255 - len);
    val[i] = s;
}

__global__ void k_morton_rows(const int* __restrict__ perm, const int* __restrict__ off, int n, int* __restrict__ inv,
                              int* __restrict__ len) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) { len[n] = 0; return; }
    const int s = perm[i];
    inv[s] = i;
    len[i] = off[s + 1] - off[s];
}

__global__ void k_morton_cols(const int* __restrict__ perm, const int* __restrict__ inv, const int* __restrict__ off,
                              const int* __restrict__ col, const int* __restrict__ moff, int n,
                              int* __restrict__ mcol) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = perm[i];
    const int e0 = off[s], e1 = off[s + 1], o = moff[i];
    for (int e = e0; e < e1; e++) mcol[o + (e - e0)] = inv[col[e]];
}

__global__ void k_gather_morton(const float4* __restrict__ p4, const int* __restrict__ perm, int n,
                                float4* __restrict__ mp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) mp[i] = p4[perm[i]];
}

__global__ void k_scatter_morton(const float4* __restrict__ mp, const int* __restrict__ perm, int n,
                                 float4* __restrict__ p4, float* __restrict__ x, float* __restrict__ y,
                                 float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 v = mp[i];
    const int s = perm[i];
    p4[s] = v;
    x[s] = v.x; y[s] = v.y; z[s] = v.z;
}

}  // namespace

// Loads the module of the general half-step kernel on the current device
// (CUDA loads kernel modules lazily, on first use, by default).
egt_status taubin_preload() {
    cudaFuncAttributes fa{};
    EGT_CUDA_TRY(cudaFuncGetAttributes(&fa, k_taubin));
    return EGT_OK;
}

egt_status taubin_launch(const float4* pin, float4* pout, const int* off, const int* col, int n, float scale,
                         cudaStream_t st) {
    k_taubin<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pin, pout, off, col, n, scale);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// One staged half-step: a persistent grid of at most one resident wave,
// launched as a programmatic dependent of the previous kernel in the stream
// (see k_taubin_tiles).
static egt_status staged_launch(egt_handle* h, const float4* pin, float4* pout, float scale, unsigned blocks,
                                cudaStream_t st) {
    const int n = (int)h->n;
    const int tiles = (n + kTile - 1) / kTile;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(std::min<unsigned>(blocks, (unsigned)tiles));
    cfg.blockDim = dim3(kTile);
    cfg.dynamicSmemBytes = kPipeSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    EGT_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_taubin_tiles, pin, pout, (const int*)h->m_off, (const int*)h->m_col,
                                    (const int*)h->t_uni, (const uint32_t*)h->t_loc, (const int*)h->t_nu,
                                    (const int*)h->t_soff, n, tiles, scale));
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

// Builds the Morton-order copy of the CSR (when the CSR changed) and gathers
// the current positions into Morton order.
static egt_status morton_prepare(egt_handle* h) {
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    const unsigned G = (unsigned)((n + 256) / 256);
    if (!h->m_perm) {
        EGT_CUDA_TRY(dev_alloc(h, &h->m_perm, sizeof(int) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_inv, sizeof(int) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_p, sizeof(float4) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_pb, sizeof(float4) * n));
        EGT_CUDA_TRY(dev_alloc(h, &h->m_off, sizeof(int) * (n + 1)));
    }
    if (h->m_version != h->csr_version) {
        int64_t nnz = 0;
        EGT_TRY(csr_nnz(h, &nnz));  // one host round trip per CSR, at set-up
        if (h->m_cap < nnz || !h->m_col) {
            if (h->m_col) dev_free(h, h->m_col);
            h->m_col = nullptr;
            EGT_CUDA_TRY(dev_alloc(h, &h->m_col, sizeof(int) * std::max<int64_t>(nnz, 1)));
            h->m_cap = std::max<int64_t>(nnz, 1);
        }
        // keys: 30-bit Morton code of the level-0 cell, below the cloud id for batches
        const bool wide = h->cloud_of != nullptr;
        const int end_bit = wide ? 30 + h->cloud_bits : 30;
        const size_t kb = wide ? sizeof(unsigned long long) : sizeof(uint32_t);
        void *kin = nullptr, *kout = nullptr;
        int *idx = nullptr, *len = nullptr;
        EGT_CUDA_TRY(cudaMallocAsync(&kin, kb * n, st));
        EGT_CUDA_TRY(cudaMallocAsync(&kout, kb * n, st));
        EGT_CUDA_TRY(cudaMallocAsync((void**)&idx, sizeof(int) * n, st));
        EGT_CUDA_TRY(cudaMallocAsync((void**)&len, sizeof(int) * (n + 1), st));
        if (wide) k_morton_keys64<<<G, 256, 0, st>>>(h->cell0, h->cloud_of, n, (unsigned long long*)kin, idx);
        else k_morton_keys<<<G, 256, 0, st>>>(h->cell0, n, (uint32_t*)kin, idx);
        EGT_LAUNCH_CHECK();
        size_t t_sort = 0, t_scan = 0;
        if (wide)
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (unsigned long long*)kin,
                                                         (unsigned long long*)kout, idx, h->m_perm, n, 0, end_bit, st));
        else
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_sort, (uint32_t*)kin, (uint32_t*)kout, idx,
                                                         h->m_perm, n, 0, end_bit, st));
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t_scan, len, h->m_off, n + 1, st));
        const int64_t tiles = (n + kTile - 1) / kTile;
        int tile_bits = 0;
        while ((int64_t(1) << tile_bits) < tiles) tile_bits++;
        size_t t_deg = 0;
        EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, t_deg, (uint32_t*)kin, (uint32_t*)kout, idx, h->m_perm,
                                                     n, 0, 8 + tile_bits, st));
        void* tmp = nullptr;
        EGT_TRY(scratch_reserve(h, std::max(std::max(t_sort, t_scan), t_deg), &tmp));
        if (wide)
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, (unsigned long long*)kin,
                                                         (unsigned long long*)kout, idx, h->m_perm, n, 0, end_bit, st));
        else
            EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, (uint32_t*)kin, (uint32_t*)kout, idx,
                                                         h->m_perm, n, 0, end_bit, st));
        // within each tile, rows by decreasing neighbour count
        k_degree_keys<<<G, 256, 0, st>>>(h->m_perm, h->csr_off, n, (uint32_t*)kin, idx);
        EGT_LAUNCH_CHECK();
        EGT_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_deg, (uint32_t*)kin, (uint32_t*)kout, idx, h->m_perm, n,
                                                     0, 8 + tile_bits, st));
        k_morton_rows<<<G, 256, 0, st>>>(h->m_perm, h->csr_off, n, h->m_inv, len);
        EGT_LAUNCH_CHECK();
        EGT_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, t_scan, len, h->m_off, n + 1, st));
        k_morton_cols<<<G, 256, 0, st>>>(h->m_perm, h->m_inv, h->csr_off, h->csr_col, h->m_off, n, h->m_col);
        EGT_LAUNCH_CHECK();
        // per-tile staged-slot tables for the staged half-step (fixed strides
        // per tile; the sizes depend only on n, so they are kept across CSRs)
        if (h->t_tiles != tiles) {
            if (h->t_uni) dev_free(h, h->t_uni);
            if (h->t_loc) dev_free(h, h->t_loc);
            if (h->t_nu) dev_free(h, h->t_nu);
            if (h->t_soff) dev_free(h, h->t_soff);
            h->t_uni = nullptr; h->t_loc = nullptr; h->t_nu = nullptr; h->t_soff = nullptr;
            h->t_tiles = 0;
            EGT_CUDA_TRY(dev_alloc(h, &h->t_uni, sizeof(int) * kUCap * tiles));
            EGT_CUDA_TRY(dev_alloc(h, &h->t_loc, sizeof(uint32_t) * kSellWords * tiles));
            EGT_CUDA_TRY(dev_alloc(h, &h->t_nu, sizeof(int) * tiles));
            EGT_CUDA_TRY(dev_alloc(h, &h->t_soff, sizeof(int) * kSoffWords * tiles));
            h->t_tiles = tiles;
        }
        EGT_CUDA_TRY(cudaMemsetAsync(h->d_counters + kCtrSpillTiles, 0, sizeof(unsigned long long), st));
        k_tile_build<<<(unsigned)tiles, kBuildThreads, 0, st>>>(h->m_off, h->m_col, n, h->t_uni, h->t_loc, h->t_nu,
                                                                 h->t_soff, h->d_counters + kCtrSpillTiles);
        EGT_LAUNCH_CHECK();
        h->tm.taubin_tiles = tiles;
        cudaFreeAsync(kin, st);
        cudaFreeAsync(kout, st);
        cudaFreeAsync(idx, st);
        cudaFreeAsync(len, st);
        h->m_version = h->csr_version;
    }
    k_gather_morton<<<G, 256, 0, st>>>(h->p4, h->m_perm, n, h->m_p);
    EGT_LAUNCH_CHECK();
    return EGT_OK;
}

egt_status run_taubin(egt_handle* h, int iters, float lambda, float mu) {
    if (iters < 0) { set_error("egt_taubin: iters must be >= 0"); return EGT_ERR_ARG; }
    if (!h->lists) { set_error("egt_taubin: no neighbour lists"); return EGT_ERR_STATE; }
    EGT_TRY(ensure_csr(h));
    cudaStream_t st = h->stream;
    const int n = (int)h->n;
    EGT_CUDA_TRY(cudaEventRecord(h->ev[6], st));
    if (iters > 0) {
        EGT_TRY(morton_prepare(h));
        // function attributes are per device: set them once on each, and size
        // the persistent grid from the occupancy they allow
        static std::atomic<uint64_t> attr_set{0};
        static std::atomic<unsigned> wave[64];
        int dev = 0;
        EGT_CUDA_TRY(cudaGetDevice(&dev));
        if (!(attr_set.load() >> (dev & 63) & 1)) {
            EGT_CUDA_TRY(cudaFuncSetAttribute(k_taubin_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kPipeSmem));
            // the whole unified L1/shared array as shared memory, so that four
            // 50-KB blocks fit on an SM
            EGT_CUDA_TRY(cudaFuncSetAttribute(k_taubin_tiles, cudaFuncAttributePreferredSharedMemoryCarveout,
                                              (int)cudaSharedmemCarveoutMaxShared));
            int sms = 0, per = 0;
            EGT_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            EGT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_taubin_tiles, kTile, kPipeSmem));
            wave[dev & 63].store((unsigned)std::max(1, sms * std::max(per, 1)));
            attr_set.fetch_or(uint64_t(1) << (dev & 63));
        }
        const unsigned blocks = wave[dev & 63].load();
        // every buffer the captured launches name
        const void* key[8] = {h->m_p, h->m_pb, h->t_uni, h->t_loc, h->t_nu, h->t_soff, h->m_off, h->m_col};
        const bool reuse = h->taubin_exec && h->taubin_iters == iters && h->taubin_lambda == lambda &&
                           h->taubin_mu == mu && h->taubin_graph_mode == h->taubin_mode &&
                           std::equal(key, key + 8, h->taubin_key);
        if (!reuse) {
            if (h->taubin_exec) { cudaGraphExecDestroy(h->taubin_exec); h->taubin_exec = nullptr; }
            // capture the 2*iters half-steps once; replays reuse the executable graph
            cudaGraph_t g = nullptr;
            cudaStream_t cap = nullptr;
            EGT_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            egt_status s = EGT_OK;
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                for (int it = 0; it < iters && s == EGT_OK; it++) {
                    if (h->taubin_mode == 0) {
                        s = staged_launch(h, h->m_p, h->m_pb, lambda, blocks, cap);
                        if (s == EGT_OK) s = staged_launch(h, h->m_pb, h->m_p, mu, blocks, cap);
                    } else {  // direct gathers (no tile staging)
                        s = taubin_launch(h->m_p, h->m_pb, h->m_off, h->m_col, n, lambda, cap);
                        if (s == EGT_OK) s = taubin_launch(h->m_pb, h->m_p, h->m_off, h->m_col, n, mu, cap);
                    }
                }
                cudaError_t e2 = cudaStreamEndCapture(cap, &g);
                if (e2 != cudaSuccess && s == EGT_OK) { set_error(cuda_msg(e2, "EndCapture", __FILE__, __LINE__)); s = EGT_ERR_CUDA; }
            } else {
                set_error(cuda_msg(e, "BeginCapture", __FILE__, __LINE__));
                s = EGT_ERR_CUDA;
            }
            if (s == EGT_OK) {
                e = cudaGraphInstantiate(&h->taubin_exec, g, 0);
                if (e != cudaSuccess) {
                    set_error(cuda_msg(e, "GraphInstantiate", __FILE__, __LINE__));
                    h->taubin_exec = nullptr;
                    s = EGT_ERR_CUDA;
                }
            }
            if (g) cudaGraphDestroy(g);
            cudaStreamDestroy(cap);
            EGT_TRY(s);
            h->taubin_iters = iters;
            h->taubin_graph_mode = h->taubin_mode;
            h->taubin_lambda = lambda;
            h->taubin_mu = mu;
            std::copy(key, key + 8, h->taubin_key);
        } else {
            // the graph's launches are counted at capture; count the replayed ones too
            for (int i = 0; i < 2 * iters; i++) count_launch();
        }
        EGT_CUDA_TRY(cudaGraphLaunch(h->taubin_exec, st));
        k_scatter_morton<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->m_p, h->m_perm, n, h->p4, h->x, h->y,
                                                                       h->z);
        EGT_LAUNCH_CHECK();
    } else {
        k_split_soa<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(h->p4, n, h->x, h->y, h->z);
        EGT_LAUNCH_CHECK();
    }
    EGT_CUDA_TRY(cudaEventRecord(h->ev[7], st));
    return EGT_OK;
}

}  // namespace egt

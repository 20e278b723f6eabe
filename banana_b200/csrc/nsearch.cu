// Uniform-grid cell sort, Morton z-sort and neighbour search (BananaCore/Banana/Grid,
// BananaCore/Banana/NeighborSearch) as standalone device entry points.
//
// Sorting is a stable LSD radix sort (8-bit digits, passes only over the key bits that
// vary): per 2048-item tile a 256-bin histogram, a digit-major exclusive scan over all
// tiles, then a scatter that ranks equal digits in input order with warp match masks.
// Stability gives the canonical order of equal keys (input order), which is what the
// reference's one-thread bucket fill produces.
#include "bnn_internal.cuh"

#include <mutex>
#include <vector>

namespace bnn {
cudaError_t exclusive_scan_u32_to_u64(const uint32_t* in, unsigned long long* out, size_t n, void* ws, cudaStream_t s);
size_t scan_workspace_bytes_u64(size_t n);

namespace {
constexpr int kRT = 256;           // threads per radix tile
constexpr int kRPer = 8;           // rounds per tile
constexpr int kRTile = kRT * kRPer;
constexpr int kWarps = kRT / 32;

template<class K> __global__ void __launch_bounds__(kRT) k_radix_hist(const K* __restrict__ keys, size_t n, int shift,
                                                                      uint32_t* __restrict__ hist, unsigned ntiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kRTile;
    for(int r = 0; r < kRPer; ++r) {
        size_t e = base + (size_t)r * kRT + threadIdx.x;
        if(e < n) atomicAdd(&h[(unsigned)((keys[e] >> shift) & 0xFF)], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template<class K> __global__ void __launch_bounds__(kRT) k_radix_scatter(const K* __restrict__ kin,
                                                                         const uint32_t* __restrict__ vin,
                                                                         K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                                         size_t n, int shift,
                                                                         const uint32_t* __restrict__ offs,
                                                                         unsigned ntiles) {
    __shared__ uint32_t runBase[256];
    __shared__ uint32_t cnt[kWarps][256];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    runBase[t] = offs[(size_t)t * ntiles + blockIdx.x];
    const size_t base = (size_t)blockIdx.x * kRTile;
    const unsigned lt = (1u << lane) - 1u;
    for(int r = 0; r < kRPer; ++r) {
#pragma unroll
        for(int q = 0; q < kWarps; ++q) cnt[q][t] = 0;
        __syncthreads();
        const size_t e = base + (size_t)r * kRT + t;
        const bool valid = e < n;
        K key = valid ? kin[e] : K(0);
        const unsigned d = valid ? (unsigned)((key >> shift) & 0xFF) : 256u;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned rank = __popc(peers & lt);
        if(valid && rank == 0) cnt[w][d] = __popc(peers);
        __syncthreads();
        if(valid) {
            uint32_t off = 0;
            for(int q = 0; q < w; ++q) off += cnt[q][d];
            const uint32_t dst = runBase[d] + off + rank;
            kout[dst] = key;
            vout[dst] = vin ? vin[e] : (uint32_t)e;
        }
        __syncthreads();
        uint32_t tot = 0;
#pragma unroll
        for(int q = 0; q < kWarps; ++q) tot += cnt[q][t];
        runBase[t] += tot;
        __syncthreads();
    }
}

template<class K> __global__ void k_key_bits(const K* __restrict__ keys, size_t n, unsigned long long* orv,
                                             unsigned long long* andv) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long o = 0, a = ~0ull;
    for(; i < n; i += (size_t)gridDim.x * blockDim.x) {
        unsigned long long k = (unsigned long long)keys[i];
        o |= k;
        a &= k;
    }
    for(int off = 16; off > 0; off >>= 1) {
        o |= __shfl_xor_sync(0xffffffffu, o, off);
        a &= __shfl_xor_sync(0xffffffffu, a, off);
    }
    if((threadIdx.x & 31) == 0) { atomicOr(orv, o); atomicAnd(andv, a); }
}

__global__ void k_iota(uint32_t* v, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) v[i] = (uint32_t)i;
}

// Grid::getCellIdx + getCellLinearizedIndex (Grid.h:108-111,156-162), clamped to the grid
__global__ void k_grid_cell_ids(const float* __restrict__ pos, uint32_t n, float b0, float b1, float b2, float cs,
                                int n0, int n1, int n2, uint32_t* __restrict__ cid, unsigned* oor) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    int c[3] = {(int)((pos[3 * p] - b0) / cs), (int)((pos[3 * p + 1] - b1) / cs), (int)((pos[3 * p + 2] - b2) / cs)};
    const int nn[3] = {n0, n1, n2};
    bool out = false;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        if(c[d] < 0) { c[d] = 0; out = true; }
        if(c[d] >= nn[d]) { c[d] = nn[d] - 1; out = true; }
    }
    if(out) atomicAdd(oor, 1u);
    cid[p] = (uint32_t)(((size_t)c[2] * n1 + c[1]) * n0 + c[0]);
}

__global__ void k_histogram(const uint32_t* __restrict__ keys, size_t n, uint32_t* __restrict__ count) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n) atomicAdd(count + keys[i], 1u);
}

// NeighborSearch::cell_index (NeighborSearch.cpp:44-52) with SHIFT_POSITION 1.2345
// (DataStructures.h:32) and inv_cell_size = float(1.0 / r)
__device__ __forceinline__ void ns_key(float x, float y, float z, float inv, int k[3]) {
    const float sh = 1.2345f;
    const float t[3] = {x - sh, y - sh, z - sh};
#pragma unroll
    for(int d = 0; d < 3; ++d) k[d] = t[d] >= 0.f ? (int)(inv * t[d]) : (int)(inv * t[d]) - 1;
}

// Morton code as m3D_e_sLUT<uint_fast64_t, uint_fast32_t> (Morton/Morton3D.h:54-66):
// 8 byte groups, each x/y/z byte bit-interleaved and shifted in by 24 bits, so only the
// three low bytes of each coordinate survive in the 64-bit code.
__device__ __forceinline__ unsigned long long spread8(unsigned b) {
    unsigned long long r = 0;
#pragma unroll
    for(int i = 0; i < 8; ++i) r |= (unsigned long long)((b >> i) & 1u) << (3 * i);
    return r;
}
__device__ __forceinline__ unsigned long long morton3d(unsigned long long x, unsigned long long y,
                                                       unsigned long long z) {
    unsigned long long ans = 0;
#pragma unroll
    for(int i = 8; i > 0; --i) {
        const unsigned sh = (unsigned)(i - 1) * 8;
        ans = (ans << 24) | (spread8((unsigned)((z >> sh) & 0xFF)) << 2) | (spread8((unsigned)((y >> sh) & 0xFF)) << 1) |
              spread8((unsigned)((x >> sh) & 0xFF));
    }
    return ans;
}

// NeighborSearch::z_value (NeighborSearch.cpp:57-67)
__global__ void k_zvalues(const float* __restrict__ pos, uint32_t n, float inv, unsigned long long* __restrict__ z) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    int k[3];
    ns_key(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], inv, k);
    unsigned long long c[3];
#pragma unroll
    for(int d = 0; d < 3; ++d) c[d] = (unsigned long long)((long long)k[d] - ((long long)INT_MIN + 1));
    z[p] = morton3d(c[0], c[1], c[2]);
}

// Hash keys of the points and their box: reduced over the block first, so the six
// words of the box see one atomic per block instead of one per warp
__global__ void __launch_bounds__(256) k_ns_keys(const float* __restrict__ pos, uint32_t n, float inv,
                                                 int* __restrict__ keys3, int* __restrict__ kmin,
                                                 int* __restrict__ kmax) {
    __shared__ int sMin[3][8], sMax[3][8];
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    int k[3] = {INT_MAX, INT_MAX, INT_MAX}, km[3] = {INT_MIN, INT_MIN, INT_MIN};
    if(p < n) {
        ns_key(pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], inv, k);
#pragma unroll
        for(int d = 0; d < 3; ++d) { keys3[3 * p + d] = k[d]; km[d] = k[d]; }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        int a = k[d], b = km[d];
        for(int off = 16; off > 0; off >>= 1) {
            a = min(a, __shfl_xor_sync(0xffffffffu, a, off));
            b = max(b, __shfl_xor_sync(0xffffffffu, b, off));
        }
        if(lane == 0) { sMin[d][w] = a; sMax[d][w] = b; }
    }
    __syncthreads();
    if(threadIdx.x < 3) {
        const int d = threadIdx.x;
        int a = INT_MAX, b = INT_MIN;
        for(int q = 0; q < (int)(blockDim.x >> 5); ++q) { a = min(a, sMin[d][q]); b = max(b, sMax[d][q]); }
        if(a != INT_MAX) atomicMin(kmin + d, a);
        if(b != INT_MIN) atomicMax(kmax + d, b);
    }
}

__global__ void k_dense_cell(const int* __restrict__ keys3, uint32_t n, const int* __restrict__ kmin, int d0, int d1,
                             uint32_t* __restrict__ cid) {
    const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= n) return;
    const int x = keys3[3 * p] - kmin[0] + 1, y = keys3[3 * p + 1] - kmin[1] + 1, z = keys3[3 * p + 2] - kmin[2] + 1;
    cid[p] = (uint32_t)(((size_t)z * d1 + y) * d0 + x);
}

__global__ void k_gather_pos(const float* __restrict__ pos, const uint32_t* __restrict__ order, uint32_t n,
                             float4* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const uint32_t p = order[i];
    out[i] = make_float4(pos[3 * (size_t)p], pos[3 * (size_t)p + 1], pos[3 * (size_t)p + 2], __uint_as_float(p));
}

// NeighborSearch::query3D (NeighborSearch.cpp:530-692) per point: every other point of the
// 27 hash cells with (dx*dx + dy*dy) + dz*dz < r^2.  One thread per point in cell-sorted
// order, so a warp shares its candidate cells.  This pass counts each point's neighbours;
// k_ns_query_write then writes them, visiting the candidates in the same order.
__global__ void __launch_bounds__(256) k_ns_count(const float4* __restrict__ sp, const uint32_t* __restrict__ scid,
                                                  uint32_t n, const uint32_t* __restrict__ cellStart, int d0, int d1,
                                                  float r2, uint32_t* __restrict__ counts) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= n) return;
    const float4 a = sp[i];
    const uint32_t self = __float_as_uint(a.w);
    const uint32_t c = scid[i];
    const size_t plane = (size_t)d0 * d1;
    uint32_t cnt = 0;
    for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy) {
            const size_t row = (size_t)((long long)c + dz * (long long)plane + dy * (long long)d0);
            const uint32_t b = cellStart[row - 1], e = cellStart[row + 2];
            for(uint32_t j = b; j < e; ++j) {
                const float4 q = sp[j];
                const uint32_t other = __float_as_uint(q.w);
                if(other == self) continue;
                const float t0 = a.x - q.x, t1 = a.y - q.y, t2 = a.z - q.z;
                const float l2 = t0 * t0 + t1 * t1 + t2 * t2;
                if(l2 < r2) ++cnt;
            }
        }
    counts[self] = cnt;
}

// The writing pass, its stores gathered per warp: each lane appends its
// neighbours to its own row of a shared-memory buffer, and as soon as one lane's row is
// full the warp writes every lane's buffered entries out, one lane's entries at a time
// (lanes k write entry k: consecutive addresses), instead of 32 lanes storing into 32
// different lists at every candidate.  The lanes walk their candidate ranges in step (the
// warp's longest range; shorter ones idle), so the warp's votes see every lane.  Each list
// holds exactly the entries k_ns_count counted, in its visiting order.
constexpr int kNsBuf = 32;   // entries a lane's buffer row holds
constexpr int kNsGroup = 4;  // candidates tested between two checks of the rows
__global__ void __launch_bounds__(256) k_ns_query_write(const float4* __restrict__ sp, const uint32_t* __restrict__ scid,
                                                        uint32_t n, const uint32_t* __restrict__ cellStart, int d0,
                                                        int d1, float r2, const unsigned long long* __restrict__ offsets,
                                                        uint32_t* __restrict__ idx) {
    __shared__ uint32_t buf[256 / 32][32][kNsBuf + 1];  // +1: a lane's row starts in its own bank
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const float4 a = live ? sp[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t self = __float_as_uint(a.w);
    const uint32_t c = live ? scid[i] : 0u;
    const size_t plane = (size_t)d0 * d1;
    const unsigned long long o = live ? offsets[self] : 0ull;
    unsigned long long written = 0;  // entries of this lane's list already in idx
    uint32_t held = 0;               // entries in this lane's buffer row
    uint32_t* row = buf[warp][lane];
    auto flush = [&]() {
        __syncwarp();
        for(int L = 0; L < 32; ++L) {
            const uint32_t cntL = __shfl_sync(full, held, L);
            const unsigned long long dst = __shfl_sync(full, o + written, L);
            if((uint32_t)lane < cntL) idx[dst + lane] = buf[warp][L][lane];
        }
        __syncwarp();
        written += held;
        held = 0;
    };
    for(int dz = -1; dz <= 1; ++dz)
        for(int dy = -1; dy <= 1; ++dy) {
            uint32_t b = 0, e = 0;
            if(live) {
                const size_t r = (size_t)((long long)c + dz * (long long)plane + dy * (long long)d0);
                b = cellStart[r - 1];
                e = cellStart[r + 2];
            }
            const uint32_t len = e - b;
            uint32_t most = len;
#pragma unroll
            for(int off = 16; off > 0; off >>= 1) most = max(most, __shfl_xor_sync(full, most, off));
            // candidates four at a time (their loads in flight together); a group adds at
            // most four entries, so the warp writes out before any row could overflow
            for(uint32_t t = 0; t < most; t += kNsGroup) {
                float4 q[kNsGroup];
#pragma unroll
                for(int u = 0; u < kNsGroup; ++u) q[u] = t + u < len ? sp[b + t + u] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for(int u = 0; u < kNsGroup; ++u) {
                    const uint32_t other = __float_as_uint(q[u].w);
                    const float t0 = a.x - q[u].x, t1 = a.y - q[u].y, t2 = a.z - q[u].z;
                    const float l2 = t0 * t0 + t1 * t1 + t2 * t2;
                    if(t + u < len && other != self && l2 < r2) row[held++] = other;
                }
                if(__any_sync(full, held > (uint32_t)(kNsBuf - kNsGroup))) flush();
            }
        }
    if(__any_sync(full, held != 0u)) flush();
}
} // namespace

// ---- host helpers -------------------------------------------------------------------
namespace {
// Temporary device memory from the device's memory pool, allocated and freed in order on
// the stream that uses it (no device-wide synchronisation, freed memory reused by the next
// call)
struct DevBuf {
    void* p = nullptr;
    cudaStream_t s = nullptr;
    ~DevBuf() { if(p) cudaFreeAsync(p, s); }
    cudaError_t alloc(size_t b, cudaStream_t st) {
        const cudaError_t e = mem_pool_setup();
        if(e != cudaSuccess) return e;
        s = st;
        return cudaMallocAsync(&p, b ? b : 1, st);
    }
    template<class T> T* as() { return (T*)p; }
};

// stable sort of keys (input order for ties); returns permutation in permOut and sorted
// keys in keysOut.  Uses only the key bits that vary.
template<class K>
int radix_sort(const K* keys, size_t n, K* keysOut, uint32_t* permOut, cudaStream_t s) {
    if(n == 0) return BNN_OK;
    DevBuf bits, k2, v2, hist, ws;
    BNN_CUDA_CHECK(bits.alloc(2 * sizeof(unsigned long long), s));
    unsigned long long init[2] = {0ull, ~0ull};
    BNN_CUDA_CHECK(cudaMemcpyAsync(bits.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    { k_key_bits<K><<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, s>>>(keys, n, bits.as<unsigned long long>(),
                                                                                   bits.as<unsigned long long>() + 1); bnn_note_launch(); }
    unsigned long long hb[2];
    BNN_CUDA_CHECK(cudaMemcpyAsync(hb, bits.p, sizeof(hb), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    const unsigned long long vary = hb[0] ^ hb[1];
    int lo = 0, hi = -1;
    if(vary) {
        lo = __builtin_ctzll(vary) & ~7;
        hi = 63 - __builtin_clzll(vary);
    }
    const unsigned ntiles = (unsigned)((n + kRTile - 1) / kRTile);
    BNN_CUDA_CHECK(k2.alloc(n * sizeof(K), s));
    BNN_CUDA_CHECK(v2.alloc(n * sizeof(uint32_t), s));
    BNN_CUDA_CHECK(hist.alloc(((size_t)256 * ntiles + 1) * sizeof(uint32_t), s));
    size_t wsb = scan_workspace_bytes((size_t)256 * ntiles);
    if(wsb) BNN_CUDA_CHECK(ws.alloc(wsb, s));
    std::vector<int> shifts;
    for(int sh = lo; sh <= hi; sh += 8) shifts.push_back(sh);
    // ping-pong so that the last pass lands in keysOut / permOut
    const K* kin = keys;
    const uint32_t* vin = nullptr;
    const int np = (int)shifts.size();
    if(np == 0) {
        BNN_CUDA_CHECK(cudaMemcpyAsync(keysOut, keys, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        { k_iota<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(permOut, n); bnn_note_launch(); }
        return BNN_OK;
    }
    for(int pi = 0; pi < np; ++pi) {
        const bool toOut = ((np - 1 - pi) % 2) == 0;
        K* kout = toOut ? keysOut : k2.as<K>();
        uint32_t* vout = toOut ? permOut : v2.as<uint32_t>();
        { k_radix_hist<K><<<ntiles, kRT, 0, s>>>(kin, n, shifts[pi], hist.as<uint32_t>(), ntiles); bnn_note_launch(); }
        BNN_CUDA_CHECK(exclusive_scan_u32(hist.as<uint32_t>(), hist.as<uint32_t>(), (size_t)256 * ntiles, ws.p, s));
        { k_radix_scatter<K><<<ntiles, kRT, 0, s>>>(kin, vin, kout, vout, n, shifts[pi], hist.as<uint32_t>(), ntiles); bnn_note_launch(); }
        BNN_CUDA_CHECK(cudaGetLastError());
        kin = kout;
        vin = vout;
    }
    return BNN_OK;
}
} // namespace
} // namespace bnn

using namespace bnn;

extern "C" int bnn_cell_sort(const float* pos_dev, uint32_t n, const float bmin[3], float cell_size,
                             const int32_t ncells[3], uint32_t* cell_id_dev, uint32_t* sorted_idx_dev,
                             uint32_t* cell_start_dev, uint32_t* out_of_range, void* stream) {
    if((n && (!pos_dev || !cell_id_dev || !sorted_idx_dev)) || !bmin || !ncells || !(cell_size > 0.f))
        return BNN_ERR_INVALID_ARGUMENT;
    for(int d = 0; d < 3; ++d) if(ncells[d] <= 0) return BNN_ERR_INVALID_ARGUMENT;
    const size_t C = (size_t)ncells[0] * ncells[1] * ncells[2];
    if(C >= 0xffffffffull) return BNN_ERR_NOT_SUPPORTED;
    cudaStream_t s = (cudaStream_t)stream;
    DevBuf oor, keysSorted;
    BNN_CUDA_CHECK(oor.alloc(sizeof(unsigned), s));
    BNN_CUDA_CHECK(cudaMemsetAsync(oor.p, 0, sizeof(unsigned), s));
    if(n) {
        { k_grid_cell_ids<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, n, bmin[0], bmin[1], bmin[2], cell_size, ncells[0],
                                                         ncells[1], ncells[2], cell_id_dev, oor.as<unsigned>()); bnn_note_launch(); }
        BNN_CUDA_CHECK(keysSorted.alloc((size_t)n * sizeof(uint32_t), s));
        int rc = radix_sort<uint32_t>(cell_id_dev, n, keysSorted.as<uint32_t>(), sorted_idx_dev, s);
        if(rc != BNN_OK) return rc;
    }
    if(cell_start_dev) {
        DevBuf cnt, ws;
        BNN_CUDA_CHECK(cnt.alloc(C * sizeof(uint32_t), s));
        BNN_CUDA_CHECK(cudaMemsetAsync(cnt.p, 0, C * sizeof(uint32_t), s));
        if(n) { k_histogram<<<(n + 255) / 256, 256, 0, s>>>(cell_id_dev, n, cnt.as<uint32_t>()); bnn_note_launch(); }
        size_t wsb = scan_workspace_bytes(C);
        if(wsb) BNN_CUDA_CHECK(ws.alloc(wsb, s));
        BNN_CUDA_CHECK(exclusive_scan_u32(cnt.as<uint32_t>(), cell_start_dev, C, ws.p, s));
    }
    unsigned h = 0;
    BNN_CUDA_CHECK(cudaMemcpyAsync(&h, oor.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    if(out_of_range) *out_of_range = h;
    return BNN_OK;
}

extern "C" int bnn_z_sort(const float* pos_dev, uint32_t n, float radius, uint64_t* zvalue_dev, uint32_t* perm_dev,
                          void* stream) {
    if((n && (!pos_dev || !zvalue_dev || !perm_dev)) || !(radius > 0.f)) return BNN_ERR_INVALID_ARGUMENT;
    if(n == 0) return BNN_OK;
    cudaStream_t s = (cudaStream_t)stream;
    const float inv = (float)(1.0 / (double)radius);
    { k_zvalues<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, n, inv, (unsigned long long*)zvalue_dev); bnn_note_launch(); }
    DevBuf sorted;
    BNN_CUDA_CHECK(sorted.alloc((size_t)n * sizeof(unsigned long long), s));
    int rc = radix_sort<unsigned long long>((const unsigned long long*)zvalue_dev, n, sorted.as<unsigned long long>(),
                                            perm_dev, s);
    if(rc != BNN_OK) return rc;
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    return BNN_OK;
}

extern "C" int bnn_neighbors(const float* pos_dev, uint32_t n, float radius, uint64_t* offsets_dev, uint32_t* idx_dev,
                             uint64_t capacity, uint64_t* total, void* stream) {
    if((n && (!pos_dev || !offsets_dev)) || !(radius > 0.f)) return BNN_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    if(n == 0) {
        BNN_CUDA_CHECK(cudaMemsetAsync(offsets_dev, 0, sizeof(uint64_t), s));
        if(total) *total = 0;
        return BNN_OK;
    }
    const float inv = (float)(1.0 / (double)radius);
    const float r2 = radius * radius;
    DevBuf keys3, kmm, cid, cidSorted, order, sp, cnt, start, ws, counts, ws64;
    BNN_CUDA_CHECK(keys3.alloc((size_t)n * 3 * sizeof(int), s));
    BNN_CUDA_CHECK(kmm.alloc(6 * sizeof(int), s));
    int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    BNN_CUDA_CHECK(cudaMemcpyAsync(kmm.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    { k_ns_keys<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, n, inv, keys3.as<int>(), kmm.as<int>(), kmm.as<int>() + 3); bnn_note_launch(); }
    int hk[6];
    BNN_CUDA_CHECK(cudaMemcpyAsync(hk, kmm.p, sizeof(hk), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    // dense key box with one empty cell of padding on every side
    const long long d0 = (long long)hk[3] - hk[0] + 3, d1 = (long long)hk[4] - hk[1] + 3, d2 = (long long)hk[5] - hk[2] + 3;
    const long long V = d0 * d1 * d2;
    if(V > (1ll << 30)) return BNN_ERR_NOT_SUPPORTED;
    BNN_CUDA_CHECK(cid.alloc((size_t)n * sizeof(uint32_t), s));
    { k_dense_cell<<<(n + 255) / 256, 256, 0, s>>>(keys3.as<int>(), n, kmm.as<int>(), (int)d0, (int)d1, cid.as<uint32_t>()); bnn_note_launch(); }
    BNN_CUDA_CHECK(cidSorted.alloc((size_t)n * sizeof(uint32_t), s));
    BNN_CUDA_CHECK(order.alloc((size_t)n * sizeof(uint32_t), s));
    int rc = radix_sort<uint32_t>(cid.as<uint32_t>(), n, cidSorted.as<uint32_t>(), order.as<uint32_t>(), s);
    if(rc != BNN_OK) return rc;
    BNN_CUDA_CHECK(sp.alloc((size_t)n * sizeof(float4), s));
    { k_gather_pos<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, order.as<uint32_t>(), n, sp.as<float4>()); bnn_note_launch(); }
    BNN_CUDA_CHECK(cnt.alloc((size_t)V * sizeof(uint32_t), s));
    BNN_CUDA_CHECK(start.alloc(((size_t)V + 1) * sizeof(uint32_t), s));
    BNN_CUDA_CHECK(cudaMemsetAsync(cnt.p, 0, (size_t)V * sizeof(uint32_t), s));
    { k_histogram<<<(n + 255) / 256, 256, 0, s>>>(cid.as<uint32_t>(), n, cnt.as<uint32_t>()); bnn_note_launch(); }
    size_t wsb = scan_workspace_bytes((size_t)V);
    if(wsb) BNN_CUDA_CHECK(ws.alloc(wsb, s));
    BNN_CUDA_CHECK(exclusive_scan_u32(cnt.as<uint32_t>(), start.as<uint32_t>(), (size_t)V, ws.p, s));
    BNN_CUDA_CHECK(counts.alloc((size_t)n * sizeof(uint32_t), s));
    { k_ns_count<<<(n + 255) / 256, 256, 0, s>>>(sp.as<float4>(), cidSorted.as<uint32_t>(), n, start.as<uint32_t>(),
                                                 (int)d0, (int)d1, r2, counts.as<uint32_t>()); bnn_note_launch(); }
    size_t wsb64 = scan_workspace_bytes_u64(n);
    if(wsb64) BNN_CUDA_CHECK(ws64.alloc(wsb64, s));
    BNN_CUDA_CHECK(exclusive_scan_u32_to_u64(counts.as<uint32_t>(), (unsigned long long*)offsets_dev, n, ws64.p, s));
    uint64_t tot = 0;
    BNN_CUDA_CHECK(cudaMemcpyAsync(&tot, offsets_dev + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    if(total) *total = tot;
    if(tot > capacity) return BNN_ERR_CAPACITY;
    if(tot && !idx_dev) return BNN_ERR_INVALID_ARGUMENT;
    { k_ns_query_write<<<(n + 255) / 256, 256, 0, s>>>(sp.as<float4>(), cidSorted.as<uint32_t>(), n, start.as<uint32_t>(),
                                                      (int)d0, (int)d1, r2, (const unsigned long long*)offsets_dev,
                                                      idx_dev); bnn_note_launch(); }
    BNN_CUDA_CHECK(cudaGetLastError());
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    return BNN_OK;
}

// ---------------------------------------------------------------------------------
// Cell sort without any device allocation.
//
// Some callers cannot allocate device memory at the moment they need a sort: an
// application whose own pool allocator has already reserved all device memory, or a loop
// on a latency budget in which cudaMalloc / cudaFree would synchronise the device and
// stall the work queued on other streams.  For them this entry point works entirely in a
// fixed scratch array compiled into the library: every GPU that loads the library holds
// kNoAllocScratchBytes (about 21 MiB) until the process exits.  Limits: at most
// kNoAllocMaxPoints points and kNoAllocMaxCells grid cells.
// ---------------------------------------------------------------------------------
namespace {
constexpr uint32_t kNoAllocMaxPoints = 1u << 20;  // 1,048,576 points
constexpr uint32_t kNoAllocMaxCells = 1u << 21;   // 2,097,152 cells (e.g. 128^3)
constexpr uint32_t kNoAllocTiles = (kNoAllocMaxPoints + kRTile - 1) / kRTile;
constexpr size_t kAlign = 256;
constexpr size_t alignUp(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }
constexpr size_t kOffCounter = 0;                                                     // out-of-range count
constexpr size_t kOffKeys0 = alignUp(kOffCounter + 16);                               // sorted keys
constexpr size_t kOffKeys1 = alignUp(kOffKeys0 + sizeof(uint32_t) * kNoAllocMaxPoints);  // ping-pong keys
constexpr size_t kOffVals1 = alignUp(kOffKeys1 + sizeof(uint32_t) * kNoAllocMaxPoints);  // ping-pong payload
constexpr size_t kOffHist = alignUp(kOffVals1 + sizeof(uint32_t) * kNoAllocMaxPoints);   // radix histogram (+1)
constexpr size_t kOffCells = alignUp(kOffHist + sizeof(uint32_t) * (256u * kNoAllocTiles + 1));  // cell counts
constexpr size_t kOffScanWs = alignUp(kOffCells + sizeof(uint32_t) * kNoAllocMaxCells);  // scan workspace
constexpr size_t kScanWsBytes = 64u * 1024u;  // >= scan_workspace_bytes of either scan, checked at run time
constexpr size_t kNoAllocScratchBytes = alignUp(kOffScanWs + kScanWsBytes);
} // namespace

static __device__ __align__(256) unsigned char g_cellSortScratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noallocMutex;
// device address of g_cellSortScratch per device ordinal, and the id of the context it
// was resolved in (a reset device gets a new context, in which the module -- and so the
// array -- can sit at another address)
void* g_noallocPtr[64] = {};
unsigned long long g_noallocCtx[64] = {};

// Id of the current context (cuCtxGetId through the runtime's driver entry point, so the
// library does not link libcuda); 0 when the driver cannot tell.
unsigned long long current_context_id() {
    using GetId = int (*)(void*, unsigned long long*);  // CUresult cuCtxGetId(CUcontext, unsigned long long*)
    static GetId fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if(cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess ||
           q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (GetId)f;
    }();
    unsigned long long id = 0;
    if(fn && fn(nullptr, &id) != 0) id = 0;
    return id;
}

// First call on a device (or in a new context of it): resolve the scratch array's device
// address with that device current.  The host-side symbol is only a stand-in and must
// never reach a kernel.
int noalloc_scratch(unsigned char** out) {
    int dev = 0;
    BNN_CUDA_CHECK(cudaGetDevice(&dev));
    if(dev < 0 || dev >= 64) return BNN_ERR_NOT_SUPPORTED;
    // 0 before the runtime made a context current: resolve (which makes it current)
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lock(g_noallocMutex);
    if(!g_noallocPtr[dev] || ctx == 0 || g_noallocCtx[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_cellSortScratch);
        if(e != cudaSuccess || !p) {
            bnn_set_error(e != cudaSuccess ? cudaGetErrorString(e) : "scratch symbol has no device address");
            return BNN_ERR_CUDA;
        }
        g_noallocPtr[dev] = p;
        g_noallocCtx[dev] = current_context_id();
    }
    *out = (unsigned char*)g_noallocPtr[dev];
    return BNN_OK;
}
} // namespace

extern "C" int bnn_cell_sort_noalloc(const float* pos_dev, uint32_t n, const float bmin[3], float cell_size,
                                     const int32_t ncells[3], uint32_t* cell_id_dev, uint32_t* sorted_idx_dev,
                                     uint32_t* cell_start_dev, uint32_t* out_of_range, void* stream) {
    if((n && (!pos_dev || !cell_id_dev || !sorted_idx_dev)) || !bmin || !ncells || !(cell_size > 0.f))
        return BNN_ERR_INVALID_ARGUMENT;
    for(int d = 0; d < 3; ++d) if(ncells[d] <= 0) return BNN_ERR_INVALID_ARGUMENT;
    const size_t C = (size_t)ncells[0] * ncells[1] * ncells[2];
    if(n > kNoAllocMaxPoints || C > kNoAllocMaxCells) {
        bnn_set_error("bnn_cell_sort_noalloc: more than 1,048,576 points or 2,097,152 cells does not fit the "
                      "fixed scratch array; use bnn_cell_sort");
        return BNN_ERR_CAPACITY;
    }
    if(scan_workspace_bytes((size_t)256 * kNoAllocTiles) > kScanWsBytes || scan_workspace_bytes(C) > kScanWsBytes)
        return BNN_ERR_CAPACITY;
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if(rc != BNN_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned* oor = (unsigned*)(scratch + kOffCounter);
    uint32_t* keys0 = (uint32_t*)(scratch + kOffKeys0);
    uint32_t* keys1 = (uint32_t*)(scratch + kOffKeys1);
    uint32_t* vals1 = (uint32_t*)(scratch + kOffVals1);
    uint32_t* hist = (uint32_t*)(scratch + kOffHist);
    uint32_t* cells = (uint32_t*)(scratch + kOffCells);
    void* scanWs = scratch + kOffScanWs;
    // the array keeps the previous call's contents: zero what is accumulated into
    BNN_CUDA_CHECK(cudaMemsetAsync(oor, 0, sizeof(unsigned), s));
    if(n) {
        { k_grid_cell_ids<<<(n + 255) / 256, 256, 0, s>>>(pos_dev, n, bmin[0], bmin[1], bmin[2], cell_size, ncells[0],
                                                         ncells[1], ncells[2], cell_id_dev, oor); bnn_note_launch(); }
        // stable LSD radix sort over the bits a cell id < C can have; ping-pong so the
        // last pass writes the caller's sorted_idx_dev
        int bits = 0;
        while(bits < 32 && ((size_t)1 << bits) < C) ++bits;
        const int passes = (bits + 7) / 8;
        const unsigned ntiles = (unsigned)((n + kRTile - 1) / kRTile);
        if(passes == 0) {
            { k_iota<<<(n + 255) / 256, 256, 0, s>>>(sorted_idx_dev, n); bnn_note_launch(); }
        }
        const uint32_t* kin = cell_id_dev;
        const uint32_t* vin = nullptr;
        for(int pi = 0; pi < passes; ++pi) {
            const bool toOut = ((passes - 1 - pi) % 2) == 0;
            uint32_t* kout = toOut ? keys0 : keys1;
            uint32_t* vout = toOut ? sorted_idx_dev : vals1;
            { k_radix_hist<uint32_t><<<ntiles, kRT, 0, s>>>(kin, n, 8 * pi, hist, ntiles); bnn_note_launch(); }
            BNN_CUDA_CHECK(exclusive_scan_u32(hist, hist, (size_t)256 * ntiles, scanWs, s));
            { k_radix_scatter<uint32_t><<<ntiles, kRT, 0, s>>>(kin, vin, kout, vout, n, 8 * pi, hist, ntiles); bnn_note_launch(); }
            kin = kout;
            vin = vout;
        }
    }
    if(cell_start_dev) {
        BNN_CUDA_CHECK(cudaMemsetAsync(cells, 0, C * sizeof(uint32_t), s));
        if(n) { k_histogram<<<(n + 255) / 256, 256, 0, s>>>(cell_id_dev, n, cells); bnn_note_launch(); }
        BNN_CUDA_CHECK(exclusive_scan_u32(cells, cell_start_dev, C, scanWs, s));
    }
    BNN_CUDA_CHECK(cudaGetLastError());
    unsigned h = 0;
    BNN_CUDA_CHECK(cudaMemcpyAsync(&h, oor, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    if(out_of_range) *out_of_range = h;
    return BNN_OK;
}

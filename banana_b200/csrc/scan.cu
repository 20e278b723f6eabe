// Device-wide exclusive prefix sums (cell histograms, active-cell numbering, neighbour
// list offsets).  Integer addition is exact, so the result does not depend on the
// block layout.
#include "bnn_internal.cuh"

#include <cstdint>
#include <type_traits>

namespace bnn {

namespace {
constexpr int kScanThreads = 256;
constexpr int kScanPer = 8;
constexpr int kScanTile = kScanThreads * kScanPer;

template<class T> __device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for(int off = 1; off < 32; off <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, v, off);
        if(lane >= off) v += o;
    }
    return v;
}

// Exclusive scan of one 2048-element tile; writes the tile total to sums[blockIdx.x] and,
// for a single-tile scan, also out[n].
template<class TI, class TO>
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(const TI* __restrict__ in, TO* __restrict__ out,
                                                             TO* __restrict__ sums, size_t n) {
    __shared__ TO warpTot[kScanThreads / 32];
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
    TO v[kScanPer];
    TO local = 0;
#pragma unroll
    for(int j = 0; j < kScanPer; ++j) {
        size_t e = base + j;
        v[j] = e < n ? (TO)in[e] : (TO)0;
        local += v[j];
    }
    TO incl = warp_incl_scan(local);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 31) warpTot[warp] = incl;
    __syncthreads();
    if(warp == 0) {
        TO w = lane < kScanThreads / 32 ? warpTot[lane] : (TO)0;
        TO wi = warp_incl_scan(w);
        if(lane < kScanThreads / 32) warpTot[lane] = wi - w;
    }
    __syncthreads();
    TO run = warpTot[warp] + incl - local;
#pragma unroll
    for(int j = 0; j < kScanPer; ++j) {
        size_t e = base + j;
        if(e < n) out[e] = run;
        run += v[j];
    }
    if(threadIdx.x == kScanThreads - 1) {
        if(sums) sums[blockIdx.x] = run;
        if(gridDim.x == 1) out[n] = run;
    }
}

template<class TO> __global__ void k_scan_add(TO* __restrict__ out, const TO* __restrict__ offs, size_t n) {
    const TO o = offs[blockIdx.x];
    const size_t base = (size_t)blockIdx.x * kScanTile;
    for(int j = threadIdx.x; j < kScanTile; j += kScanThreads) {
        size_t e = base + j;
        if(e < n) out[e] += o;
    }
}

template<class TO> __global__ void k_copy_total(TO* out, size_t n, const TO* sumsScan, size_t nb) { out[n] = sumsScan[nb]; }

// ---- reduce-then-scan of 32-bit inputs -----------------------------------------------
// Three launches for any n: the tile sums (one 16384-element tile per block), their scan,
// and the tiles' scans with the tile offsets added.  The last pass reads its tile again,
// from L2 for arrays up to a few tens of MB (the cell histograms, the active-cell flags),
// so DRAM sees about one read and one write of the array.  Every load and store is 16
// bytes: tile element (j * kRtsThreads + t) * 4 + c belongs to thread t, load j, lane c
// of the vector, so each warp instruction moves 512 contiguous bytes.
constexpr int kRtsThreads = 512;
constexpr int kRtsVec = 8;
constexpr int kRtsTile = kRtsThreads * kRtsVec * 4;
constexpr int kRtsWarps = kRtsThreads / 32;

__device__ __forceinline__ void rts_load(const uint32_t* __restrict__ in, size_t n, size_t tb, uint4 q[kRtsVec]) {
#pragma unroll
    for(int j = 0; j < kRtsVec; ++j) {
        const size_t e = tb + ((size_t)j * kRtsThreads + threadIdx.x) * 4;
        if(e + 4 <= n) {
            q[j] = *reinterpret_cast<const uint4*>(in + e);
        } else {
            q[j].x = e < n ? in[e] : 0u;
            q[j].y = e + 1 < n ? in[e + 1] : 0u;
            q[j].z = e + 2 < n ? in[e + 2] : 0u;
            q[j].w = 0u;
        }
    }
}

template<class TO> __device__ __forceinline__ TO quad_sum(const uint4& v) {
    return (TO)v.x + (TO)v.y + (TO)v.z + (TO)v.w;
}

// The sum of tile `tile` to *dst (all threads of the block take part)
template<class TO>
__device__ __forceinline__ void rts_sums_body(const uint32_t* __restrict__ in, size_t n, size_t tile,
                                              TO* __restrict__ dst) {
    __shared__ TO wsum[kRtsWarps];
    uint4 q[kRtsVec];
    rts_load(in, n, tile * kRtsTile, q);
    TO t = 0;
#pragma unroll
    for(int j = 0; j < kRtsVec; ++j) t += quad_sum<TO>(q[j]);
#pragma unroll
    for(int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 0) wsum[warp] = t;
    __syncthreads();
    if(warp == 0) {
        TO v = lane < kRtsWarps ? wsum[lane] : (TO)0;
#pragma unroll
        for(int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if(lane == 0) *dst = v;
    }
}

template<class TO>
__global__ void __launch_bounds__(kRtsThreads) k_rts_sums(const uint32_t* __restrict__ in, TO* __restrict__ sums,
                                                          size_t n) {
    rts_sums_body(in, n, blockIdx.x, sums + blockIdx.x);
}

template<class TO> __device__ __forceinline__ void store_quad(TO* __restrict__ out, size_t e, size_t n, TO a, TO b,
                                                              TO c, TO d);
template<> __device__ __forceinline__ void store_quad<uint32_t>(uint32_t* __restrict__ out, size_t e, size_t n,
                                                                uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    if(e + 4 <= n) {
        *reinterpret_cast<uint4*>(out + e) = make_uint4(a, b, c, d);
    } else {
        if(e < n) out[e] = a;
        if(e + 1 < n) out[e + 1] = b;
        if(e + 2 < n) out[e + 2] = c;
    }
}
template<> __device__ __forceinline__ void store_quad<unsigned long long>(unsigned long long* __restrict__ out, size_t e,
                                                                          size_t n, unsigned long long a,
                                                                          unsigned long long b, unsigned long long c,
                                                                          unsigned long long d) {
    if(e + 4 <= n) {
        *reinterpret_cast<ulonglong2*>(out + e) = make_ulonglong2(a, b);
        *reinterpret_cast<ulonglong2*>(out + e + 2) = make_ulonglong2(c, d);
    } else {
        if(e < n) out[e] = a;
        if(e + 1 < n) out[e + 1] = b;
        if(e + 2 < n) out[e + 2] = c;
    }
}

// Exclusive scan of tile `tile` plus `base` into out; `totalOut`, if given, gets base plus
// the tile's sum
template<class TO>
__device__ __forceinline__ void rts_final_body(const uint32_t* __restrict__ in, TO* __restrict__ out, TO base,
                                               size_t n, size_t tile, TO* __restrict__ totalOut) {
    __shared__ TO part[kRtsVec * kRtsWarps];  // warp totals in tile order: load j, then warp
    const size_t tb = tile * kRtsTile;
    uint4 q[kRtsVec];
    rts_load(in, n, tb, q);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    TO sum[kRtsVec], inc[kRtsVec];
#pragma unroll
    for(int j = 0; j < kRtsVec; ++j) {
        sum[j] = quad_sum<TO>(q[j]);
        inc[j] = warp_incl_scan(sum[j]);
        if(lane == 31) part[j * kRtsWarps + warp] = inc[j];
    }
    __syncthreads();
    if(warp == 0) {
        constexpr int kPer = kRtsVec * kRtsWarps / 32;
        TO v[kPer];
        TO loc = 0;
#pragma unroll
        for(int k = 0; k < kPer; ++k) { v[k] = part[lane * kPer + k]; loc += v[k]; }
        const TO li = warp_incl_scan(loc);
        TO run = li - loc;
#pragma unroll
        for(int k = 0; k < kPer; ++k) { part[lane * kPer + k] = run; run += v[k]; }
        if(totalOut && lane == 31) *totalOut = base + li;
    }
    __syncthreads();
#pragma unroll
    for(int j = 0; j < kRtsVec; ++j) {
        const TO r = base + part[j * kRtsWarps + warp] + inc[j] - sum[j];
        const TO r1 = r + (TO)q[j].x, r2 = r1 + (TO)q[j].y, r3 = r2 + (TO)q[j].z;
        store_quad<TO>(out, tb + ((size_t)j * kRtsThreads + threadIdx.x) * 4, n, r, r1, r2, r3);
    }
}

// offs: the exclusive scan of the tile sums; the last tile writes the total to out[n]
template<class TO>
__global__ void __launch_bounds__(kRtsThreads, sizeof(TO) == 4 ? 2 : 1) k_rts_final(const uint32_t* __restrict__ in, TO* __restrict__ out,
                                                           const TO* __restrict__ offs, size_t n) {
    rts_final_body(in, out, offs[blockIdx.x], n, blockIdx.x, blockIdx.x == gridDim.x - 1 ? out + n : nullptr);
}

template<class TO> size_t ws_bytes(size_t n) {
    size_t nb = (n + kScanTile - 1) / kScanTile;
    if(nb <= 1) return 0;
    size_t here = ((nb + 1) * 2 * sizeof(TO) + 255) & ~size_t(255);
    return here + ws_bytes<TO>(nb);
}

template<class TI, class TO> cudaError_t scan_impl(const TI* in, TO* out, size_t n, void* ws, cudaStream_t s) {
    size_t nb = (n + kScanTile - 1) / kScanTile;
    if(n == 0) return cudaMemsetAsync(out, 0, sizeof(TO), s);
    if(nb == 1) {
        { k_scan_tile<TI, TO><<<1, kScanThreads, 0, s>>>(in, out, nullptr, n); bnn_note_launch(); }
        return cudaGetLastError();
    }
    if(std::is_same<TI, uint32_t>::value && ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 15u) == 0) {
        // reduce-then-scan: fewer tiles than the scan below, so its workspace holds them
        const size_t nt = (n + kRtsTile - 1) / kRtsTile;
        TO* sums = (TO*)ws;
        TO* sumsScan = sums + (nt + 1);
        const size_t here = ((nt + 1) * 2 * sizeof(TO) + 255) & ~size_t(255);
        const uint32_t* in32 = reinterpret_cast<const uint32_t*>(in);
        { k_rts_sums<TO><<<(unsigned)nt, kRtsThreads, 0, s>>>(in32, sums, n); bnn_note_launch(); }
        cudaError_t e = scan_impl<TO, TO>(sums, sumsScan, nt, (char*)ws + here, s);
        if(e != cudaSuccess) return e;
        { k_rts_final<TO><<<(unsigned)nt, kRtsThreads, 0, s>>>(in32, out, sumsScan, n); bnn_note_launch(); }
        return cudaGetLastError();
    }
    TO* sums = (TO*)ws;
    TO* sumsScan = sums + (nb + 1);
    size_t here = ((nb + 1) * 2 * sizeof(TO) + 255) & ~size_t(255);
    void* rest = (char*)ws + here;
    { k_scan_tile<TI, TO><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, sums, n); bnn_note_launch(); }
    cudaError_t e = scan_impl<TO, TO>(sums, sumsScan, nb, rest, s);
    if(e != cudaSuccess) return e;
    { k_scan_add<TO><<<(unsigned)nb, kScanThreads, 0, s>>>(out, sumsScan, n); bnn_note_launch(); }
    { k_copy_total<TO><<<1, 1, 0, s>>>(out, n, sumsScan, nb); bnn_note_launch(); }
    return cudaGetLastError();
}

// ---- batched segments ----------------------------------------------------------------
// Segment q: tiles tiles[q] .. tiles[q+1]-1 of the launch, kScanSegTile elements each (at
// least one, so an empty segment still gets its total 0).  Its tile sums go to ws[0..nb],
// their scan to ws[nb+1 ..] (the layout of scan_impl's first level).
static_assert(kRtsTile == kScanSegTile, "segment tiles are the reduce-then-scan tiles");
// tile sums of every segment of more than one tile
__global__ void __launch_bounds__(kRtsThreads) kb_rts_sums(const ScanSeg* __restrict__ segs,
                                                           const unsigned* __restrict__ tiles, int nseg) {
    int q;
    const Blk b = seg_blk(tiles, nseg, q);
    if(b.n <= 1) return;
    const ScanSeg sg = segs[q];
    rts_sums_body<uint32_t>(sg.in, sg.n, b.x, sg.ws + b.x);
}
// Exclusive scan of m <= kScanTile values by one block, continuing from `carry` (updated to
// the running total; every thread gets it)
__device__ __forceinline__ void scan_chunk_carry(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                 unsigned m, uint32_t& carry) {
    __shared__ uint32_t warpTot[kScanThreads / 32];
    __shared__ uint32_t sTotal;
    const unsigned base = threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    uint32_t local = 0;
#pragma unroll
    for(int j = 0; j < kScanPer; ++j) {
        v[j] = base + j < m ? in[base + j] : 0u;
        local += v[j];
    }
    const uint32_t incl = warp_incl_scan(local);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(lane == 31) warpTot[warp] = incl;
    __syncthreads();
    if(warp == 0) {
        const uint32_t w = lane < kScanThreads / 32 ? warpTot[lane] : 0u;
        const uint32_t wi = warp_incl_scan(w);
        if(lane < kScanThreads / 32) warpTot[lane] = wi - w;
        if(lane == kScanThreads / 32 - 1) sTotal = wi;
    }
    __syncthreads();
    uint32_t run = carry + warpTot[warp] + incl - local;
#pragma unroll
    for(int j = 0; j < kScanPer; ++j) {
        if(base + j < m) out[base + j] = run;
        run += v[j];
    }
    carry += sTotal;
    __syncthreads();
}
// one block per segment: scan of its tile sums, and the total
__global__ void __launch_bounds__(kScanThreads) kb_scan_sums(const ScanSeg* __restrict__ segs,
                                                             const unsigned* __restrict__ tiles) {
    const ScanSeg sg = segs[blockIdx.x];
    const unsigned nb = __ldg(tiles + blockIdx.x + 1) - __ldg(tiles + blockIdx.x);
    if(nb <= 1) return;
    uint32_t* sumsScan = sg.ws + (nb + 1);
    uint32_t carry = 0;
    for(unsigned b0 = 0; b0 < nb; b0 += kScanTile)
        scan_chunk_carry(sg.ws + b0, sumsScan + b0, min(nb - b0, (unsigned)kScanTile), carry);
    if(threadIdx.x == 0) sg.out[sg.n] = carry;
}
// the tiles' scans from their offsets (kb_scan_sums); a one-tile segment writes its total
__global__ void __launch_bounds__(kRtsThreads, 2) kb_rts_final(const ScanSeg* __restrict__ segs,
                                                            const unsigned* __restrict__ tiles, int nseg) {
    int q;
    const Blk b = seg_blk(tiles, nseg, q);
    const ScanSeg sg = segs[q];
    const uint32_t base = b.n > 1 ? sg.ws[(b.n + 1) + b.x] : 0u;
    rts_final_body<uint32_t>(sg.in, sg.out, base, sg.n, b.x, b.n == 1 ? sg.out + sg.n : nullptr);
}
} // namespace

cudaError_t batched_exclusive_scan_u32(const ScanSeg* segs, const unsigned* tiles, int nseg, unsigned totalTiles,
                                       cudaStream_t s) {
    if(nseg == 0 || totalTiles == 0) return cudaSuccess;
    { kb_rts_sums<<<totalTiles, kRtsThreads, 0, s>>>(segs, tiles, nseg); bnn_note_launch(); }
    { kb_scan_sums<<<(unsigned)nseg, kScanThreads, 0, s>>>(segs, tiles); bnn_note_launch(); }
    { kb_rts_final<<<totalTiles, kRtsThreads, 0, s>>>(segs, tiles, nseg); bnn_note_launch(); }
    return cudaGetLastError();
}
size_t scan_workspace_bytes(size_t n) { return ws_bytes<uint32_t>(n); }
size_t scan_workspace_bytes_u64(size_t n) { return ws_bytes<unsigned long long>(n); }

cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, size_t n, void* ws, cudaStream_t s) {
    return scan_impl<uint32_t, uint32_t>(in, out, n, ws, s);
}
cudaError_t exclusive_scan_u32_to_u64(const uint32_t* in, unsigned long long* out, size_t n, void* ws, cudaStream_t s) {
    return scan_impl<uint32_t, unsigned long long>(in, out, n, ws, s);
}

} // namespace bnn

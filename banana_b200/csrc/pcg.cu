// Matrix-free Jacobi PCG for the 7-point pressure system (PCGSolver::solve_precond,
// BananaCore/Banana/LinearAlgebra/LinearSolvers/PCGSolver.cpp:143-199).
//
// Rows are the fluid cells in linear-cell order.  Per row: diag (float), 1/diag, and six
// neighbour row indices in ascending column order (-z,-y,-x,+x,+y,+z; -1 = none), stored
// as six planes nbr[q*n + r].  Every off-diagonal equals -dt (face weight 1), so the
// matrix is never materialised.
//
// One iteration is two kernels, both in the canonical 2048-row chunk layout so their
// FP64 dot products are bit-reproducible:
//   spmv   : s = z + beta*s_old formed on the fly (double buffered), q = A s, partial s.q;
//            the last block forms alpha = rho / (s.q)
//   update : x += alpha s, r -= alpha q, max|r|, z = D^-1 r, partial z.r; the last block
//            tests max|r| < tol*max|b| and forms beta
// Scalars live in DevState; once `done` is set every later launch returns at once, so
// the host can queue iterations in batches and only look at `done` between batches.
#include "bnn_internal.cuh"

#include <vector>

namespace bnn {

template<class VT> struct Sc;
template<> struct Sc<float> {
    __device__ static float alpha(const DevState* s) { return s->alpha; }
    __device__ static float beta(const DevState* s) { return s->beta; }
    __device__ static void set_alpha(DevState* s, double a) { s->alpha = (float)a; }
    __device__ static void set_beta(DevState* s, double b) { s->beta = (float)b; }
    __device__ static float tol(const DevState* s) { return s->tol; }
    __device__ static void set_tol(DevState* s, float t) { s->tol = t; }
    __device__ static void set_resid(DevState* s, float r) { s->resid = r; s->resid64 = r; }
};
template<> struct Sc<double> {
    __device__ static double alpha(const DevState* s) { return s->alpha64; }
    __device__ static double beta(const DevState* s) { return s->beta64; }
    __device__ static void set_alpha(DevState* s, double a) { s->alpha64 = a; }
    __device__ static void set_beta(DevState* s, double b) { s->beta64 = b; }
    __device__ static double tol(const DevState* s) { return s->tol64; }
    __device__ static void set_tol(DevState* s, double t) { s->tol64 = t; }
    __device__ static void set_resid(DevState* s, double r) { s->resid64 = r; s->resid = (float)r; }
};

template<class VT> __device__ __forceinline__ VT vabs(VT x) { return x < VT(0) ? -x : x; }

template<class VT> __device__ __forceinline__ VT block_max_t(VT v, VT* sm) {
    const int t = threadIdx.x;
    sm[t] = v;
    __syncthreads();
    for(int off = 128; off > 0; off >>= 1) {
        if(t < off) { VT o = sm[t + off]; sm[t] = sm[t] > o ? sm[t] : o; }
        __syncthreads();
    }
    VT r = sm[0];
    __syncthreads();
    return r;
}
template<class VT> __device__ __forceinline__ VT reduce_max_t(const VT* part, int nch, VT* sm) {
    VT acc = VT(0);
    for(int c = threadIdx.x; c < nch; c += kLanes) { VT o = __ldcg(part + c); acc = acc > o ? acc : o; }
    return block_max_t(acc, sm);
}

// r = rhs, x = 0, z = D^-1 r, rho = z.r, resid = max|r|, tol = tolFactor * resid
template<class VT>
__global__ void __launch_bounds__(kLanes) k_pcg_init(int n, const float* __restrict__ rhsF, const VT* __restrict__ rhsV,
                                                     VT* __restrict__ x, VT* __restrict__ r, VT* __restrict__ z,
                                                     const VT* __restrict__ invd, double* __restrict__ part,
                                                     VT* __restrict__ partMax, DevState* st, VT tolFactor,
                                                     unsigned maxIter) {
    __shared__ double smd[kLanes];
    __shared__ VT smv[kLanes];
    const size_t base = (size_t)blockIdx.x * kChunk + threadIdx.x;
    double acc = 0.0;
    VT m = VT(0);
#pragma unroll
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const VT rv = rhsV ? rhsV[e] : (VT)rhsF[e];
            r[e] = rv;
            x[e] = VT(0);
            const VT a = vabs(rv);
            m = m > a ? m : a;
            const VT zv = invd[e] * rv;
            z[e] = zv;
            acc = acc + (double)zv * (double)rv;
        }
    }
    const double bs = block_sum_256(acc, smd);
    const VT bm = block_max_t(m, smv);
    if(threadIdx.x == 0) { part[blockIdx.x] = bs; partMax[blockIdx.x] = bm; }
    if(last_block(&st->counter0)) {
        const int nch = gridDim.x;
        const double rho = reduce_partials(part, nch, smd);
        const VT resid = reduce_max_t(partMax, nch, smv);
        if(threadIdx.x == 0) {
            st->counter0 = 0;
            st->iter = 0;
            st->max_iter = maxIter;
            st->done = 0;
            st->success = 0;
            Sc<VT>::set_resid(st, resid);
            tolFactor = fmax(tolFactor, VT(1e-30));
            if(resid < (VT)FLT_MIN) {
                st->done = 1; st->success = 1;
            } else {
                Sc<VT>::set_tol(st, tolFactor * resid);
                if(rho < (double)FLT_MIN || isnan(rho)) { st->done = 1; st->success = 0; }
                st->rho = rho;
            }
            if(maxIter == 0 && !st->done) { st->done = 1; st->success = 0; }
        }
    }
}

template<class VT>
__device__ __forceinline__ VT s_of(const VT* __restrict__ z, const VT* __restrict__ sOld, VT beta, bool first, int e) {
    return first ? z[e] : z[e] + beta * sOld[e];
}

// s = z + beta*s_old; q = A s (column-ordered sum); partial s.q; last block: alpha
template<class VT>
__global__ void __launch_bounds__(kLanes) k_pcg_spmv(int n, const VT* __restrict__ z, const VT* __restrict__ sOld,
                                                     VT* __restrict__ sNew, VT* __restrict__ q,
                                                     const float* __restrict__ diag, const int32_t* __restrict__ nbr,
                                                     VT negoff, double* __restrict__ part, DevState* st, int first) {
    __shared__ double smd[kLanes];
    if(*(volatile unsigned*)&st->done) return;
    const VT beta = first ? VT(0) : Sc<VT>::beta(st);
    const bool fst = first != 0;
    const size_t base = (size_t)blockIdx.x * kChunk + threadIdx.x;
    double acc = 0.0;
#pragma unroll 2
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const int32_t n0 = nbr[e], n1 = nbr[(size_t)n + e], n2 = nbr[2 * (size_t)n + e];
            const int32_t n3 = nbr[3 * (size_t)n + e], n4 = nbr[4 * (size_t)n + e], n5 = nbr[5 * (size_t)n + e];
            const float dg = diag[e];
            const VT se = s_of(z, sOld, beta, fst, (int)e);
            VT t = VT(0);
            if(n0 >= 0) t += negoff * s_of(z, sOld, beta, fst, n0);
            if(n1 >= 0) t += negoff * s_of(z, sOld, beta, fst, n1);
            if(n2 >= 0) t += negoff * s_of(z, sOld, beta, fst, n2);
            if(dg != 0.f) t += (VT)dg * se;
            if(n3 >= 0) t += negoff * s_of(z, sOld, beta, fst, n3);
            if(n4 >= 0) t += negoff * s_of(z, sOld, beta, fst, n4);
            if(n5 >= 0) t += negoff * s_of(z, sOld, beta, fst, n5);
            sNew[e] = se;
            q[e] = t;
            acc = acc + (double)se * (double)t;
        }
    }
    const double bs = block_sum_256(acc, smd);
    if(threadIdx.x == 0) part[blockIdx.x] = bs;
    if(last_block(&st->counter1)) {
        const double tmp = reduce_partials(part, gridDim.x, smd);
        if(threadIdx.x == 0) {
            st->counter1 = 0;
            st->tmp = tmp;
            if(tmp < (double)FLT_MIN) {
                st->iter = st->iter + 1;
                st->done = 1;
                st->success = 1;
            } else {
                Sc<VT>::set_alpha(st, st->rho / tmp);
            }
        }
    }
}

// x += alpha s; r -= alpha q; max|r|; z = D^-1 r; partial z.r; last block: test and beta
template<class VT>
__global__ void __launch_bounds__(kLanes) k_pcg_update(int n, VT* __restrict__ x, VT* __restrict__ r,
                                                       VT* __restrict__ z, const VT* __restrict__ sNew,
                                                       const VT* __restrict__ q, const VT* __restrict__ invd,
                                                       double* __restrict__ part, VT* __restrict__ partMax,
                                                       DevState* st) {
    __shared__ double smd[kLanes];
    __shared__ VT smv[kLanes];
    if(*(volatile unsigned*)&st->done) return;
    const VT alpha = Sc<VT>::alpha(st);
    const size_t base = (size_t)blockIdx.x * kChunk + threadIdx.x;
    double acc = 0.0;
    VT m = VT(0);
#pragma unroll
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            x[e] += alpha * sNew[e];
            const VT rv = r[e] + (-alpha) * q[e];
            r[e] = rv;
            const VT a = vabs(rv);
            m = m > a ? m : a;
            const VT zv = invd[e] * rv;
            z[e] = zv;
            acc = acc + (double)zv * (double)rv;
        }
    }
    const double bs = block_sum_256(acc, smd);
    const VT bm = block_max_t(m, smv);
    if(threadIdx.x == 0) { part[blockIdx.x] = bs; partMax[blockIdx.x] = bm; }
    if(last_block(&st->counter2)) {
        const int nch = gridDim.x;
        const double rhoNew = reduce_partials(part, nch, smd);
        const VT resid = reduce_max_t(partMax, nch, smv);
        if(threadIdx.x == 0) {
            st->counter2 = 0;
            st->iter = st->iter + 1;
            Sc<VT>::set_resid(st, resid);
            if(resid < Sc<VT>::tol(st)) {
                st->done = 1;
                st->success = 1;
            } else {
                Sc<VT>::set_beta(st, rhoNew / st->rho);
                st->rho = rhoNew;
                if(st->iter >= st->max_iter) {
                    st->done = 1;
                    st->success = 0;
                    atomicOr(&st->flags, BNN_FLAG_PCG_MAXITER);
                }
            }
        }
    }
}

// ---- iterative refinement helpers -------------------------------------------------
// x64 = 0, r64 = b, outer_bmax = outer_res = max|b|
__global__ void __launch_bounds__(kLanes) k_ir_init(int n, const float* __restrict__ b, double* __restrict__ x64,
                                                    double* __restrict__ r64, double* __restrict__ partMax,
                                                    DevState* st) {
    __shared__ double sm[kLanes];
    const size_t base = (size_t)blockIdx.x * kChunk + threadIdx.x;
    double m = 0.0;
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const double bv = (double)b[e];
            x64[e] = 0.0;
            r64[e] = bv;
            const double a = vabs(bv);
            m = m > a ? m : a;
        }
    }
    const double bm = block_max_t(m, sm);
    if(threadIdx.x == 0) partMax[blockIdx.x] = bm;
    if(last_block(&st->counter3)) {
        const double mx = reduce_max_t(partMax, gridDim.x, sm);
        if(threadIdx.x == 0) { st->counter3 = 0; st->outer_bmax = mx; st->outer_res = mx; }
    }
}
// r32 = (float) r64
__global__ void k_ir_to_f32(int n, const double* __restrict__ r64, float* __restrict__ r32) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) r32[e] = (float)r64[e];
}
__global__ void k_ir_accumulate(int n, double* __restrict__ x64, const float* __restrict__ d) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) x64[e] = x64[e] + (double)d[e];
}
// r64 = b - A x64 in FP64, outer_res = max|r64|
__global__ void __launch_bounds__(kLanes) k_ir_residual(int n, const float* __restrict__ b,
                                                        const double* __restrict__ x64, double* __restrict__ r64,
                                                        const float* __restrict__ diag,
                                                        const int32_t* __restrict__ nbr, double negoff,
                                                        double* __restrict__ partMax, DevState* st) {
    __shared__ double sm[kLanes];
    const size_t base = (size_t)blockIdx.x * kChunk + threadIdx.x;
    double m = 0.0;
    for(int j = 0; j < kPerLane; ++j) {
        const size_t e = base + (size_t)j * kLanes;
        if(e < (size_t)n) {
            const int32_t nn[6] = {nbr[e], nbr[(size_t)n + e], nbr[2 * (size_t)n + e], nbr[3 * (size_t)n + e],
                                   nbr[4 * (size_t)n + e], nbr[5 * (size_t)n + e]};
            double t = 0.0;
            if(nn[0] >= 0) t += negoff * x64[nn[0]];
            if(nn[1] >= 0) t += negoff * x64[nn[1]];
            if(nn[2] >= 0) t += negoff * x64[nn[2]];
            if(diag[e] != 0.f) t += (double)diag[e] * x64[e];
            if(nn[3] >= 0) t += negoff * x64[nn[3]];
            if(nn[4] >= 0) t += negoff * x64[nn[4]];
            if(nn[5] >= 0) t += negoff * x64[nn[5]];
            const double rv = (double)b[e] - t;
            r64[e] = rv;
            const double a = vabs(rv);
            m = m > a ? m : a;
        }
    }
    const double bm = block_max_t(m, sm);
    if(threadIdx.x == 0) partMax[blockIdx.x] = bm;
    if(last_block(&st->counter3)) {
        const double mx = reduce_max_t(partMax, gridDim.x, sm);
        if(threadIdx.x == 0) { st->counter3 = 0; st->outer_res = mx; }
    }
}
__global__ void k_inv_diag64(int n, const float* __restrict__ diag, double* __restrict__ inv) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) inv[e] = diag[e] != 0.f ? 1.0 / (double)diag[e] : 0.0;
}
__global__ void k_f32_to_f64(int n, const float* __restrict__ a, double* __restrict__ b) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) b[e] = (double)a[e];
}
__global__ void k_d64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(e < (size_t)n) b[e] = (float)a[e];
}

// ---------------------------------------------------------------------------------
// Host driver
// ---------------------------------------------------------------------------------

int pcg_reserve(PcgWork& w, int n, bool fp64) {
    if(n <= w.cap && (!fp64 || w.x64)) return BNN_OK;
    if(n > w.cap) {
        pcg_release(w);
        const int cap = (int)(n * 1.25) + 4096;
        const size_t nch = ((size_t)cap + kChunk - 1) / kChunk + 1;
        BNN_CUDA_CHECK(cudaMalloc(&w.x, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.r, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.z, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.s0, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.s1, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.q, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.d32, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.r32, cap * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.part, nch * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.partMaxF, nch * sizeof(float)));
        BNN_CUDA_CHECK(cudaMalloc(&w.partMaxD, nch * sizeof(double)));
        w.cap = cap;
    }
    if(fp64 && !w.x64) {
        BNN_CUDA_CHECK(cudaMalloc(&w.x64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.r64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.z64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.s064, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.s164, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.q64, w.cap * sizeof(double)));
        BNN_CUDA_CHECK(cudaMalloc(&w.inv64, w.cap * sizeof(double)));
    }
    return BNN_OK;
}

void pcg_release(PcgWork& w) {
    for(void* p : {(void*)w.x, (void*)w.r, (void*)w.z, (void*)w.s0, (void*)w.s1, (void*)w.q, (void*)w.d32, (void*)w.r32,
                   (void*)w.part, (void*)w.partMaxF, (void*)w.partMaxD, (void*)w.x64, (void*)w.r64, (void*)w.z64,
                   (void*)w.s064, (void*)w.s164, (void*)w.q64, (void*)w.inv64})
        if(p) cudaFree(p);
    w = PcgWork();
}

// Runs one PCG solve (VT vectors).  Iterations are queued in batches; between batches the
// host reads `done` from pinned memory.  Returns BNN status; solution in x (VT).
template<class VT>
static int pcg_solve_t(int n, const float* rhsF, const VT* rhsV, const float* diag, const VT* invd,
                       const int32_t* nbr, VT negoff, VT tolFactor, unsigned maxIter, VT* x, VT* r, VT* z, VT* s0,
                       VT* s1, VT* q, double* part, VT* partMax, DevState* dst, DevState* hst, cudaStream_t s,
                       PcgOutcome& out) {
    const unsigned nch = (unsigned)((n + kChunk - 1) / kChunk);
    if(n == 0) { out = PcgOutcome(); out.success = 1; return BNN_OK; }
    k_pcg_init<VT><<<nch, kLanes, 0, s>>>(n, rhsF, rhsV, x, r, z, invd, part, partMax, dst, tolFactor, maxIter);
    BNN_CUDA_CHECK(cudaGetLastError());
    unsigned it = 0;
    unsigned batch = 4;
    for(;;) {
        for(unsigned b = 0; b < batch && it < maxIter; ++b, ++it) {
            VT* sOld = (it % 2 == 0) ? s1 : s0;
            VT* sNew = (it % 2 == 0) ? s0 : s1;
            k_pcg_spmv<VT><<<nch, kLanes, 0, s>>>(n, z, sOld, sNew, q, diag, nbr, negoff, part, dst, it == 0 ? 1 : 0);
            k_pcg_update<VT><<<nch, kLanes, 0, s>>>(n, x, r, z, sNew, q, invd, part, partMax, dst);
        }
        BNN_CUDA_CHECK(cudaGetLastError());
        BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        BNN_CUDA_CHECK(cudaStreamSynchronize(s));
        if(hst->done || it >= maxIter) break;
        if(batch < 32) batch *= 2;
    }
    out.iterations = hst->iter;
    out.success = hst->success;
    out.residual = sizeof(VT) == 8 ? hst->resid64 : (double)hst->resid;
    return BNN_OK;
}

// mode: BNN_PCG_FP32 / FP64 / REFINED.  Pressure written to `pressure` (float, n).
int pcg_solve(PcgWork& w, int n, const float* rhs, const float* diag, const float* invd, const int32_t* nbr, float dt,
              int mode, float tol, unsigned maxIter, float innerTol, float outerTol, float* pressure, double* x64out,
              DevState* dst, DevState* hst, cudaStream_t s, PcgOutcome& out) {
    int rc = pcg_reserve(w, n, mode != BNN_PCG_FP32);
    if(rc != BNN_OK) return rc;
    const unsigned nb = (unsigned)((n + 255) / 256);
    const unsigned nch = (unsigned)((n + kChunk - 1) / kChunk);
    out = PcgOutcome();
    if(mode == BNN_PCG_FP32) {
        rc = pcg_solve_t<float>(n, rhs, nullptr, diag, invd, nbr, -(1.0f * dt), tol, maxIter, w.x, w.r, w.z, w.s0,
                                w.s1, w.q, w.part, w.partMaxF, dst, hst, s, out);
        if(rc != BNN_OK) return rc;
        if(n > 0) BNN_CUDA_CHECK(cudaMemcpyAsync(pressure, w.x, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        if(x64out && n > 0) k_f32_to_f64<<<nb, 256, 0, s>>>(n, w.x, x64out);
        return BNN_OK;
    }
    if(mode == BNN_PCG_FP64) {
        if(n > 0) k_inv_diag64<<<nb, 256, 0, s>>>(n, diag, w.inv64);
        rc = pcg_solve_t<double>(n, rhs, nullptr, diag, w.inv64, nbr, -(double)(1.0f * dt), (double)tol, maxIter,
                                 w.x64, w.r64, w.z64, w.s064, w.s164, w.q64, w.part, w.partMaxD, dst, hst, s, out);
        if(rc != BNN_OK) return rc;
        if(n > 0) k_d64_to_f32<<<nb, 256, 0, s>>>(n, w.x64, pressure);
        if(x64out && n > 0)
            BNN_CUDA_CHECK(cudaMemcpyAsync(x64out, w.x64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        return BNN_OK;
    }
    // refined: FP64 outer residual and solution, FP32 inner solves
    if(n == 0) { out.success = 1; return BNN_OK; }
    k_ir_init<<<nch, kLanes, 0, s>>>(n, rhs, w.x64, w.r64, w.partMaxD, dst);
    BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    BNN_CUDA_CHECK(cudaStreamSynchronize(s));
    const double bmax = hst->outer_bmax;
    unsigned total = 0, outer = 0;
    const unsigned maxOuter = 60;
    double res = bmax;
    bool ok = bmax < (double)FLT_MIN;
    while(!ok && outer < maxOuter) {
        if(res < (double)outerTol * bmax) { ok = true; break; }
        k_ir_to_f32<<<nb, 256, 0, s>>>(n, w.r64, w.r32);
        PcgOutcome inner;
        rc = pcg_solve_t<float>(n, w.r32, nullptr, diag, invd, nbr, -(1.0f * dt), innerTol, maxIter, w.d32, w.r, w.z,
                                w.s0, w.s1, w.q, w.part, w.partMaxF, dst, hst, s, inner);
        if(rc != BNN_OK) return rc;
        total += inner.iterations;
        k_ir_accumulate<<<nb, 256, 0, s>>>(n, w.x64, w.d32);
        k_ir_residual<<<nch, kLanes, 0, s>>>(n, rhs, w.x64, w.r64, diag, nbr, (double)(-(1.0f * dt)), w.partMaxD, dst);
        BNN_CUDA_CHECK(cudaMemcpyAsync(hst, dst, sizeof(DevState), cudaMemcpyDeviceToHost, s));
        BNN_CUDA_CHECK(cudaStreamSynchronize(s));
        res = hst->outer_res;
        ++outer;
        if(total >= maxIter) break;
    }
    if(!ok && res < (double)outerTol * bmax) ok = true;
    out.iterations = total;
    out.outer = outer;
    out.residual = res;
    out.success = ok ? 1 : 0;
    k_d64_to_f32<<<nb, 256, 0, s>>>(n, w.x64, pressure);
    if(x64out) BNN_CUDA_CHECK(cudaMemcpyAsync(x64out, w.x64, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return BNN_OK;
}

} // namespace bnn

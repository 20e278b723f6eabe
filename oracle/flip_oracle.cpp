// =====================================================================================
//  TEST INFRASTRUCTURE ONLY -- the oracle.
//
//  A CPU restatement, in plain C++, of the reference's 3D FLIP step (Banana,
//  Simulation/ParticleSolvers/PICFluid) together with its scalar PCG solver
//  (BananaCore/Banana/LinearAlgebra) and its uniform-grid cell sort / neighbour search
//  (BananaCore/Banana/{Grid,NeighborSearch}).  Only tests/, __graft_entry__.smoke() and
//  bench.py's CPU-baseline leg load this library, and only as the checker or as the
//  timed CPU baseline; the CUDA product never links or calls it.
//
//  Parity status.  The reference cannot be compiled here (its glm / json / spdlog / Catch
//  submodules are empty and TBB ships only as a prebuilt binary), so this file follows
//  the reference sources line by line; every function cites the file:line it restates.
//  The only known-answer vectors the reference's own tests hold for this path are the
//  Grid checks in BananaCore/Banana/Grid/_Grid.Test.hpp:29-57 (pinned in
//  tests/test_oracle_golden.py) and the set-equality methodology of
//  BananaCore/Banana/NeighborSearch/_NeighborSearch.Test.hpp:119-212 (restated as the
//  neighbour tests).  The FLIP step and the PCG solve have no reference golden vectors:
//  they are pinned by this restatement plus analytic checks (parity unpinned by the
//  reference's own tests).
//
//  Determinism.  The reference reduces with TBB (nondeterministic join order), splats
//  P2G with CAS float atomics and buckets cells under spinlocks, so it has no single
//  bit-exact answer.  This restatement runs those loops serially in particle-array
//  order, which is what the reference computes with one TBB thread.  Two orders are
//  offered for the PCG reductions:
//    * REDUCE_REFERENCE : RealType accumulators, serial left-to-right order (the
//                         reference's ParallelObjects::DotProduct run on one thread);
//    * REDUCE_CANONICAL : FP64 accumulation in fixed 2048-element chunks, 256 lanes per
//                         chunk, each lane summing 8 strided elements, then a halving
//                         tree; chunk partials reduced the same way.  This is the order
//                         the CUDA kernels use, so the two agree bit for bit (FLIP's P2G
//                         also takes the kernels' order in this mode, below).
//  Particles are re-ordered by a stable counting sort on the cell index before each
//  P2G (the reference's Grid::collectIndexToCells + getParticleIdxSortedByCell +
//  sortData, run on one thread, BananaCore/Banana/Grid/Grid.cpp:92-114,283-309).  In the
//  reference mode P2G then sums serially in that particle order (the reference on one
//  thread); in the canonical mode FLIP's P2G sums each face in the CUDA kernel's
//  two-level order (per-cell partials in id order, added in (y, z, x)-major cell order;
//  see mapP2GCanonical).  particle ids travel with the particles so the caller always sees
//  the original order.
//
//  Compile with -ffp-contract=off (no fused multiply-add): every float operation is
//  then a single IEEE-rounded operation, as in the reference built for SSE.
// =====================================================================================
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ----------------------------------------------------------------------------------
// Scalar helpers (BananaCore/Banana/Utils/MathHelpers.h)
// ----------------------------------------------------------------------------------
template<class R> static inline R smin(R a, R b) { return (b < a) ? b : a; } // std::min
template<class R> static inline R smax(R a, R b) { return (a < b) ? b : a; } // std::max

// MathHelpers::get_barycentric(x, i, f, i_low, i_high)  (MathHelpers.h:516-530)
template<class R>
static inline void get_barycentric(R x, int& i, R& f, int i_low, int i_high) {
    R s = std::floor(x);
    i   = static_cast<int>(s);
    if(i < i_low) {
        i = i_low;
        f = 0;
    } else if(i > i_high - 2) {
        i = i_high - 2;
        f = 1;
    } else {
        f = (R)(x - s);
    }
}

// MathHelpers::lerp / bilerp / trilerp  (MathHelpers.h:549-573)
template<class R> static inline R lerp(R v0, R v1, R f) { return (R(1.0) - f) * v0 + f * v1; }
template<class R> static inline R bilerp(R v00, R v10, R v01, R v11, R fx, R fy) {
    return lerp(lerp(v00, v10, fx), lerp(v01, v11, fx), fy);
}
template<class R>
static inline R trilerp(R v000, R v100, R v010, R v110, R v001, R v101, R v011, R v111, R fx, R fy, R fz) {
    return lerp(bilerp(v000, v100, v010, v110, fx, fy), bilerp(v001, v101, v011, v111, fx, fy), fz);
}

// MathHelpers::fraction_inside(left, right)  (MathHelpers.h:823-838)
template<class R> static inline R fraction_inside(R l, R r) {
    if(l < 0 && r < 0) return R(1.0);
    if(l < 0 && r >= 0) return l / (l - r);
    if(l >= 0 && r < 0) return r / (r - l);
    return R(0);
}

template<class R> struct V3 {
    R x, y, z;
    R& operator[](int d) { return d == 0 ? x : (d == 1 ? y : z); }
    R operator[](int d) const { return d == 0 ? x : (d == 1 ? y : z); }
};
// glm::dot for vec3 evaluates (x*x + y*y) + z*z
template<class R> static inline R length2(R x, R y, R z) { return (x * x + y * y) + z * z; }

template<class T> struct Arr3 {
    int sx = 0, sy = 0, sz = 0;
    std::vector<T> d;
    void resize(int x, int y, int z, T v) {
        sx = x; sy = y; sz = z;
        d.assign((size_t)x * y * z, v);
    }
    // Array<3,T> layout (k*Sy + j)*Sx + i  (BananaCore/Banana/Array/Array.h:276)
    inline size_t lin(int i, int j, int k) const { return ((size_t)k * sy + j) * sx + i; }
    inline T& operator()(int i, int j, int k) { return d[lin(i, j, k)]; }
    inline T operator()(int i, int j, int k) const { return d[lin(i, j, k)]; }
    size_t size() const { return d.size(); }
};

// ----------------------------------------------------------------------------------
// Canonical FP64 reduction (the CUDA kernels' order); see the file header.
// ----------------------------------------------------------------------------------
static constexpr int kChunk = 2048;
static constexpr int kLanes = 256;
// pcg_mode: BNN_PCG_* in the low bits, the flag for the single-reduction form
static constexpr int kPcgModeMask = 0x0f;
static constexpr int kPcgSingleReduction = 0x10;

static double tree256(double* s) {
    for(int off = kLanes / 2; off > 0; off >>= 1)
        for(int t = 0; t < off; ++t) s[t] = s[t] + s[t + off];
    return s[0];
}

template<class A, class B>
static double dot_canonical(const A* a, const B* b, size_t n) {
    size_t nch = (n + kChunk - 1) / kChunk;
    std::vector<double> part(nch);
#pragma omp parallel for schedule(static)
    for(long long c = 0; c < (long long)nch; ++c) {
        double s[kLanes];
        for(int t = 0; t < kLanes; ++t) {
            double acc = 0.0;
            for(int j = 0; j < kChunk / kLanes; ++j) {
                size_t e = (size_t)c * kChunk + (size_t)j * kLanes + t;
                if(e < n) acc = acc + (double)a[e] * (double)b[e];
            }
            s[t] = acc;
        }
        part[c] = tree256(s);
    }
    double s[kLanes];
    for(int t = 0; t < kLanes; ++t) {
        double acc = 0.0;
        for(size_t c = t; c < nch; c += kLanes) acc = acc + part[c];
        s[t] = acc;
    }
    return tree256(s);
}

// ParallelBLAS::dotProduct (ParallelHelpers/ParallelBLAS.h:40-48) with the
// ParallelObjects::DotProduct<1> body (ParallelObjects.h:110-124) run on one thread.
template<class R>
static R dot_reference(const R* a, const R* b, size_t n, int nthreads) {
    R res = 0;
    if(nthreads <= 1) {
        for(size_t i = 0; i < n; ++i) res += a[i] * b[i];
        return res;
    }
#pragma omp parallel for reduction(+ : res) schedule(static)
    for(long long i = 0; i < (long long)n; ++i) res += a[i] * b[i];
    return res;
}

// ParallelSTL::maxAbs + ParallelObjects::MaxAbs<1> (ParallelSTL.h:73-79, ParallelObjects.h:252-272)
template<class R> static R max_abs(const R* x, size_t n) {
    R res = 0;
    for(size_t i = 0; i < n; ++i) {
        R t = std::abs(x[i]);
        res = res > t ? res : t;
    }
    return res;
}

// ----------------------------------------------------------------------------------
// Parameters shared with the ctypes wrapper (layout must match oracle.py)
// ----------------------------------------------------------------------------------
extern "C" {
struct orc_params {
    float    box_min[3];            // SimulationDomainBox BoxMin (before padding)
    float    box_max[3];            // SimulationDomainBox BoxMax
    float    cell_size;             // CellSize
    uint32_t n_expand_cells;        // NExpandCells
    float    cfl_factor;            // CFLFactor
    float    min_timestep;          // MinTimestep
    float    max_timestep;          // MaxTimestep
    float    frame_duration;        // FrameDuration
    float    pic_flip_ratio;        // PIC_FLIP_ratio
    float    cg_relative_tolerance; // CGRelativeTolerance
    uint32_t max_cg_iteration;      // MaxCGIteration
    uint32_t advection_steps;       // AdvectionSteps
    int32_t  reduce_mode;           // 0 reference order, 1 canonical FP64 order
    int32_t  pcg_mode;              // 0 FP32 vectors, 1 FP64 vectors, 2 FP32 inner + FP64 refinement;
                                    // | 0x10: single-reduction form (else PCGSolver's step order)
    int32_t  preconditioner;        // 0 Jacobi, 1 MICCL0, 2 MICCL0_SYMMETRIC
    float    refine_tolerance;      // outer tolerance for pcg_mode 2 (max-norm, relative)
    float    refine_inner_tolerance;// inner FP32 tolerance for pcg_mode 2
    int32_t  sort_each_step;        // 1: stable cell sort before each P2G
    int32_t  nthreads;              // 1: deterministic serial; >1: OpenMP timed mode
    int32_t  solver_kind;           // 0 FLIP, 1 APIC, 2 AFLIP, 3 PIC
    int32_t  apply_gravity;         // GlobalParameters ApplyGravity
    int32_t  correct_position;      // CorrectPosition
    float    repulsive_force_stiffness; // RepulsiveForceStiffness
    float    ratio_cell_size_p_radius;  // RatioCellSizePRadius
};

struct orc_step_stats {
    double   dt;
    double   frame_time;
    uint32_t frame_finished;
    uint32_t pcg_iterations;
    double   pcg_residual;
    uint32_t pcg_success;
    uint32_t n_active;
    uint32_t outer_iterations;
    uint32_t zero_phi_cells;
    double   t_move, t_sort, t_p2g, t_extrap, t_sdf, t_system, t_solve, t_update, t_g2p;
};
}

// ----------------------------------------------------------------------------------
// Sparse matrix in the reference's form: per-row column-sorted entries
// (SparseMatrix.cpp:87-96 addElement with insertPairSorted) then CSR
// (FixedSparseMatrix::constructFromSparseMatrix, SparseMatrix.cpp:198-217).
// ----------------------------------------------------------------------------------
struct CSR {
    uint32_t n = 0;
    std::vector<uint32_t> rowStart, colIndex;
    std::vector<float> colValueF;
    std::vector<double> colValueD;
};

template<class R> struct RowBuilder {
    // up to 7 entries per row
    uint32_t col[8];
    R val[8];
    int cnt = 0;
    void add(uint32_t c, R v) {
        for(int k = 0; k < cnt; ++k) {
            if(col[k] == c) { val[k] += v; return; }
        }
        int pos = cnt;
        while(pos > 0 && col[pos - 1] > c) { col[pos] = col[pos - 1]; val[pos] = val[pos - 1]; --pos; }
        col[pos] = c; val[pos] = v; ++cnt;
    }
};

// FixedSparseMatrix::multiply (SparseMatrix.cpp:222-235): sum in column-sorted order
template<class VT, class MT>
static void spmv(const CSR& A, const std::vector<MT>& vals, const VT* x, VT* y, int nthreads) {
#pragma omp parallel for schedule(static) if(nthreads > 1)
    for(long long i = 0; i < (long long)A.n; ++i) {
        VT t = 0;
        for(uint32_t j = A.rowStart[i]; j < A.rowStart[i + 1]; ++j) t += (VT)vals[j] * x[A.colIndex[j]];
        y[i] = t;
    }
}

// ----------------------------------------------------------------------------------
// PCG (BananaCore/Banana/LinearAlgebra/LinearSolvers/PCGSolver.cpp:143-469)
// ----------------------------------------------------------------------------------
struct PCGResult { uint32_t iterations = 0; double residual = 0; bool success = false; uint32_t outer = 0; };

// SparseColumnLowerFactor (PCGSolver.h:30-45)
template<class R> struct LowerFactor {
    std::vector<R> invDiag, colValue, aDiag;
    std::vector<uint32_t> colIndex, colStart;
};

// formPreconditioner_Symmetric_MICC0L0 (PCGSolver.cpp:398-466) and
// formPreconditioner_MICC0L0 (PCGSolver.cpp:294-394) on the row-sorted matrix.
template<class R>
static void form_ic(const CSR& A, const std::vector<R>& vals, LowerFactor<R>& L, bool symmetric,
                    R MICCL0Param = R(0.97), R minDiagonalRatio = R(0.25)) {
    uint32_t n = A.n;
    L.invDiag.assign(n, 0); L.aDiag.assign(n, 0); L.colStart.assign(n + 1, 0);
    L.colValue.clear(); L.colIndex.clear();
    for(uint32_t i = 0; i < n; ++i) {
        L.colStart[i] = (uint32_t)L.colIndex.size();
        for(uint32_t j = A.rowStart[i]; j < A.rowStart[i + 1]; ++j) {
            if(A.colIndex[j] > i) { L.colIndex.push_back(A.colIndex[j]); L.colValue.push_back(vals[j]); }
            else if(A.colIndex[j] == i) { L.invDiag[i] = L.aDiag[i] = vals[j]; }
        }
    }
    L.colStart[n] = (uint32_t)L.colIndex.size();
    for(uint32_t k = 0; k < n; ++k) {
        if(L.aDiag[k] < std::numeric_limits<R>::min()) continue;
        if(L.invDiag[k] < minDiagonalRatio * L.aDiag[k]) L.invDiag[k] = R(1.0) / std::sqrt(L.aDiag[k]);
        else L.invDiag[k] = R(1.0) / std::sqrt(L.invDiag[k]);
        for(uint32_t p = L.colStart[k]; p < L.colStart[k + 1]; ++p) L.colValue[p] *= L.invDiag[k];
        for(uint32_t p = L.colStart[k]; p < L.colStart[k + 1]; ++p) {
            uint32_t j = L.colIndex[p];
            R multiplier = L.colValue[p];
            if(symmetric) {
                L.invDiag[j] -= multiplier * L.colValue[p];
                uint32_t a = p + 1, b = L.colStart[j], as = L.colStart[k + 1], bs = L.colStart[j + 1];
                while(a < as && b < bs) {
                    if(L.colIndex[b] == L.colIndex[a]) { L.colValue[b] -= multiplier * L.colValue[a]; ++a; ++b; }
                    else if(L.colIndex[b] < L.colIndex[a]) ++b;
                    else ++a;
                }
            } else {
                R missing = 0;
                uint32_t a = L.colStart[k];
                uint32_t b = 0;
                uint32_t rowjBeg = A.rowStart[j], rowjLen = A.rowStart[j + 1] - A.rowStart[j];
                while(a < L.colStart[k + 1] && L.colIndex[a] < j) {
                    while(b < rowjLen) {
                        uint32_t cj = A.colIndex[rowjBeg + b];
                        if(cj < L.colIndex[a]) ++b;
                        else if(cj == L.colIndex[a]) break;
                        else { missing += L.colValue[a]; break; }
                    }
                    ++a;
                }
                if(a < L.colStart[k + 1] && L.colIndex[a] == j) L.invDiag[j] -= multiplier * L.colValue[a];
                ++a;
                b = L.colStart[j];
                while(a < L.colStart[k + 1] && b < L.colStart[j + 1]) {
                    if(L.colIndex[b] < L.colIndex[a]) ++b;
                    else if(L.colIndex[b] == L.colIndex[a]) { L.colValue[b] -= multiplier * L.colValue[a]; ++a; ++b; }
                    else { missing += L.colValue[a]; ++a; }
                }
                while(a < L.colStart[k + 1]) { missing += L.colValue[a]; ++a; }
                L.invDiag[j] -= MICCL0Param * multiplier * missing;
            }
        }
    }
}

// solveLower + solveLower_TransposeInPlace (PCGSolver.cpp:243-269)
template<class R> static void apply_ic(const LowerFactor<R>& L, const std::vector<R>& rhs, std::vector<R>& res) {
    uint32_t n = (uint32_t)L.invDiag.size();
    res = rhs;
    for(uint32_t i = 0; i < n; ++i) {
        res[i] *= L.invDiag[i];
        for(uint32_t j = L.colStart[i]; j < L.colStart[i + 1]; ++j) res[L.colIndex[j]] -= L.colValue[j] * res[i];
    }
    if(n == 0) return;
    uint32_t i = n;
    do {
        --i;
        for(uint32_t j = L.colStart[i]; j < L.colStart[i + 1]; ++j) res[i] -= L.colValue[j] * res[L.colIndex[j]];
        res[i] *= L.invDiag[i];
    } while(i > 0);
}

// PCGSolver::solve_precond in the reference's arithmetic: RealType vectors, RealType
// scalars, reference-order dot products (PCGSolver.cpp:143-199).
template<class R>
static PCGResult pcg_reference(const CSR& A, const std::vector<R>& vals, const std::vector<R>& rhs, std::vector<R>& x,
                               R tolFactor, uint32_t maxIters, int precond, int nthreads) {
    PCGResult out;
    size_t n = A.n;
    tolFactor = std::fmax(tolFactor, R(1e-30));
    x.assign(n, 0);
    std::vector<R> r = rhs, z(n), s(n);
    R resid = max_abs(r.data(), n);
    out.residual = resid;
    if(resid < std::numeric_limits<R>::min()) { out.iterations = 0; out.success = true; return out; }
    R tol = tolFactor * resid;
    std::vector<R> jac;
    LowerFactor<R> L;
    if(precond == 0) {
        jac.assign(n, 0);
        for(size_t i = 0; i < n; ++i)
            for(uint32_t j = A.rowStart[i]; j < A.rowStart[i + 1]; ++j)
                if(A.colIndex[j] == i) jac[i] = R(1.0) / vals[j];
    } else {
        form_ic(A, vals, L, precond == 2);
    }
    auto apply = [&](const std::vector<R>& in, std::vector<R>& outv) {
        if(precond == 0) { for(size_t i = 0; i < n; ++i) outv[i] = jac[i] * in[i]; }
        else apply_ic(L, in, outv);
    };
    apply(r, z);
    R rho = dot_reference(z.data(), r.data(), n, nthreads);
    if(rho < std::numeric_limits<R>::min() || std::isnan(rho)) { out.iterations = 0; out.success = false; return out; }
    s = z;
    for(uint32_t it = 0; it < maxIters; ++it) {
        spmv(A, vals, s.data(), z.data(), nthreads);
        R tmp = dot_reference(s.data(), z.data(), n, nthreads);
        if(tmp < std::numeric_limits<R>::min()) { out.iterations = it + 1; out.success = true; return out; }
        R alpha = rho / tmp;
        for(size_t i = 0; i < n; ++i) x[i] += alpha * s[i];
        for(size_t i = 0; i < n; ++i) r[i] += (-alpha) * z[i];
        resid = max_abs(r.data(), n);
        out.residual = resid;
        if(resid < tol) { out.iterations = it + 1; out.success = true; return out; }
        apply(r, z);
        R rho_new = dot_reference(z.data(), r.data(), n, nthreads);
        R beta = rho_new / rho;
        for(size_t i = 0; i < n; ++i) z[i] += beta * s[i];
        s.swap(z);
        rho = rho_new;
    }
    out.iterations = maxIters; out.success = false;
    return out;
}

// Jacobi PCG with the CUDA kernels' arithmetic: VT vectors (float or double), FP64
// canonical-order reductions, alpha/beta formed in FP64 and rounded to VT.
template<class VT>
static PCGResult pcg_canonical(const CSR& A, const std::vector<float>& vals, const std::vector<float>& diag,
                               const std::vector<VT>& rhs, std::vector<VT>& x, VT tolFactor, uint32_t maxIters) {
    PCGResult out;
    size_t n = A.n;
    tolFactor = std::fmax(tolFactor, VT(1e-30));
    x.assign(n, 0);
    std::vector<VT> r = rhs, z(n), s(n), inv(n);
    for(size_t i = 0; i < n; ++i) inv[i] = diag[i] != 0 ? VT(1.0) / (VT)diag[i] : VT(0);
    VT resid = max_abs(r.data(), n);
    out.residual = resid;
    if(resid < (VT)std::numeric_limits<float>::min()) { out.success = true; return out; }
    VT tol = tolFactor * resid;
    for(size_t i = 0; i < n; ++i) z[i] = inv[i] * r[i];
    double rho = dot_canonical(z.data(), r.data(), n);
    if(rho < (double)std::numeric_limits<float>::min() || std::isnan(rho)) { out.success = false; return out; }
    s = z;
    for(uint32_t it = 0; it < maxIters; ++it) {
        spmv(A, vals, s.data(), z.data(), 1);
        double tmp = dot_canonical(s.data(), z.data(), n);
        if(tmp < (double)std::numeric_limits<float>::min()) { out.iterations = it + 1; out.success = true; return out; }
        VT alpha = (VT)(rho / tmp);
        for(size_t i = 0; i < n; ++i) {
            x[i] += alpha * s[i];
            r[i] += (-alpha) * z[i];
        }
        resid = max_abs(r.data(), n);
        out.residual = resid;
        if(resid < tol) { out.iterations = it + 1; out.success = true; return out; }
        for(size_t i = 0; i < n; ++i) z[i] = inv[i] * r[i];
        double rho_new = dot_canonical(z.data(), r.data(), n);
        VT beta = (VT)(rho_new / rho);
        for(size_t i = 0; i < n; ++i) s[i] = z[i] + beta * s[i];
        rho = rho_new;
    }
    out.iterations = maxIters; out.success = false;
    return out;
}

// The single-reduction form of the same Jacobi PCG (Chronopoulos & Gear) with the CUDA
// kernel's arithmetic: u = D^-1 r, w = A u, gamma = (r, u) and delta = (w, u) in one
// canonical FP64 reduction; beta = gamma / gamma_old and alpha = gamma / (delta -
// beta gamma / alpha_old) in FP64, rounded to VT; p = u + beta p, s = w + beta s,
// x += alpha p, r -= alpha s.  Same iterates as pcg_canonical in exact arithmetic
// (PCGSolver::solve_precond, PCGSolver.cpp:143-199), same stopping rule on max|r|.
template<class VT>
static PCGResult pcg_canonical_cg1(const CSR& A, const std::vector<float>& vals, const std::vector<float>& diag,
                                   const std::vector<VT>& rhs, std::vector<VT>& x, VT tolFactor, uint32_t maxIters) {
    PCGResult out;
    const size_t n = A.n;
    tolFactor = std::fmax(tolFactor, VT(1e-30));
    x.assign(n, 0);
    std::vector<VT> r = rhs, u(n), w(n), p(n, VT(0)), s(n, VT(0)), inv(n);
    for(size_t i = 0; i < n; ++i) inv[i] = diag[i] != 0 ? VT(1.0) / (VT)diag[i] : VT(0);
    for(size_t i = 0; i < n; ++i) u[i] = inv[i] * r[i];
    spmv(A, vals, u.data(), w.data(), 1);
    VT resid = max_abs(r.data(), n);
    out.residual = resid;
    double gamma = dot_canonical(u.data(), r.data(), n);
    double delta = dot_canonical(w.data(), u.data(), n);
    if(resid < (VT)std::numeric_limits<float>::min()) { out.success = true; return out; }
    const VT tol = tolFactor * resid;
    if(gamma < (double)std::numeric_limits<float>::min() || std::isnan(gamma)) { out.success = false; return out; }
    double gammaOld = 0.0, a64Old = 0.0;
    bool first = true;
    for(uint32_t it = 0; it < maxIters; ++it) {
        double b64 = 0.0, den = delta;
        if(!first) {
            b64 = gamma / gammaOld;
            den = delta - (b64 * gamma) / a64Old;
        }
        if(den < (double)std::numeric_limits<float>::min()) { out.iterations = it + 1; out.success = true; return out; }
        const double a64 = gamma / den;
        const VT alpha = (VT)a64, beta = (VT)b64;
        for(size_t i = 0; i < n; ++i) {
            const VT uOld = inv[i] * r[i];
            p[i] = first ? uOld : uOld + beta * p[i];
            s[i] = first ? w[i] : w[i] + beta * s[i];
            x[i] = x[i] + alpha * p[i];
            r[i] = r[i] + (-alpha) * s[i];
            u[i] = inv[i] * r[i];
        }
        spmv(A, vals, u.data(), w.data(), 1);
        resid = max_abs(r.data(), n);
        out.residual = resid;
        const double gNew = dot_canonical(u.data(), r.data(), n);
        const double dNew = dot_canonical(w.data(), u.data(), n);
        if(resid < tol) { out.iterations = it + 1; out.success = true; return out; }
        gammaOld = gamma;
        gamma = gNew;
        delta = dNew;
        a64Old = a64;
        first = false;
    }
    out.iterations = maxIters; out.success = false;
    return out;
}

// The canonical solve of either form: PCGSolver's two-reduction step order, or the
// single-reduction one.
template<class VT>
static PCGResult pcg_canonical_any(const CSR& A, const std::vector<float>& vals, const std::vector<float>& diag,
                                   const std::vector<VT>& rhs, std::vector<VT>& x, VT tolFactor, uint32_t maxIters,
                                   bool twoReductions) {
    return twoReductions ? pcg_canonical<VT>(A, vals, diag, rhs, x, tolFactor, maxIters)
                         : pcg_canonical_cg1<VT>(A, vals, diag, rhs, x, tolFactor, maxIters);
}

// Mixed-precision iterative refinement: FP64 outer residual and solution, FP32 inner
// Jacobi PCG (canonical arithmetic) on the residual.  Stops when
// max|b - A x| < outerTol * max|b|.
static PCGResult pcg_refined(const CSR& A, const std::vector<float>& vals, const std::vector<float>& diag,
                             const std::vector<float>& rhs, std::vector<double>& x, float innerTol, double outerTol,
                             uint32_t maxIters, bool twoReductions, uint32_t maxOuter = 60) {
    PCGResult out;
    size_t n = A.n;
    std::vector<double> vals64(vals.begin(), vals.end());
    std::vector<double> b(rhs.begin(), rhs.end()), r64 = b, ax(n);
    x.assign(n, 0.0);
    if(n == 0) { out.success = true; return out; }
    const double bmax = max_abs(b.data(), n);
    double res = bmax;
    bool ok = bmax < (double)std::numeric_limits<float>::min();
    uint32_t total = 0, outer = 0;
    std::vector<float> r32(n), d;
    while(!ok && outer < maxOuter) {
        if(res < outerTol * bmax) { ok = true; break; }
        for(size_t i = 0; i < n; ++i) r32[i] = (float)r64[i];
        PCGResult inner = pcg_canonical_any<float>(A, vals, diag, r32, d, innerTol, maxIters, twoReductions);
        total += inner.iterations;
        for(size_t i = 0; i < n; ++i) x[i] = x[i] + (double)d[i];
        spmv(A, vals64, x.data(), ax.data(), 1);
        for(size_t i = 0; i < n; ++i) r64[i] = b[i] - ax[i];
        res = max_abs(r64.data(), n);
        ++outer;
        if(total >= maxIters) break;
    }
    if(!ok && res < outerTol * bmax) ok = true;
    out.iterations = total;
    out.outer = outer;
    out.residual = res;
    out.success = ok;
    return out;
}

// ----------------------------------------------------------------------------------
// The FLIP step
// ----------------------------------------------------------------------------------
// One boundary object (the layout of bnn_boundary_object): BoundaryObject over a Box or
// Sphere geometry (Simulation/SimulationObjects/BoundaryObject.h:41-60), with its current
// world-to-object map (GeometryObject::invTransform, GeometryObjects.cpp:231-238)
struct orc_boundary_object {
    int32_t geometry;          // 0 box, 1 sphere
    int32_t dynamic;
    float   box_min[3];
    float   box_max[3];
    float   inv_transform[12]; // rows of a 3x4 affine map
    float   uniform_scale;
    int32_t transformed;
};
template<class R> struct OObj {
    int geometry = 0, transformed = 0;
    R bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0}, M[12] = {0}, scale = 1;
};

// MathHelpers::fraction_inside(bl, br, tl, tr) (MathHelpers.h:821-900): area fraction of a
// square inside (negative) from its corner values, the corners walked as bl, br, tr, tl
template<class R> static R fraction_inside4(R bl, R br, R tl, R tr) {
    int inside = (bl < 0 ? 1 : 0) + (tl < 0 ? 1 : 0) + (br < 0 ? 1 : 0) + (tr < 0 ? 1 : 0);
    R l[4] = {bl, br, tr, tl};
    auto cycle = [&l]() { R t = l[0]; for(int i = 0; i < 3; ++i) l[i] = l[i + 1]; l[3] = t; };
    if(inside == 4) return R(1.0);
    if(inside == 3) {
        while(l[0] < 0) cycle();
        R side0 = R(1.0) - fraction_inside(l[0], l[3]);
        R side1 = R(1.0) - fraction_inside(l[0], l[1]);
        return R(1.0) - R(0.5) * side0 * side1;
    }
    if(inside == 2) {
        while(l[0] >= 0 || !(l[1] < 0 || l[2] < 0)) cycle();
        if(l[1] < 0) {
            R left = fraction_inside(l[0], l[3]);
            R right = fraction_inside(l[1], l[2]);
            return R(0.5) * (left + right);
        }
        R mid = R(0.25) * (l[0] + l[1] + l[2] + l[3]);
        if(mid < 0) {
            R area = 0;
            R side1 = R(1.0) - fraction_inside(l[0], l[3]);
            R side3 = R(1.0) - fraction_inside(l[2], l[3]);
            area += R(0.5) * side1 * side3;
            R side2 = R(1.0) - fraction_inside(l[2], l[1]);
            R side0 = R(1.0) - fraction_inside(l[0], l[1]);
            area += R(0.5) * side0 * side2;
            return R(1.0) - area;
        }
        R area = 0;
        R side0 = fraction_inside(l[0], l[1]);
        R side1 = fraction_inside(l[0], l[3]);
        area += R(0.5) * side0 * side1;
        R side2 = fraction_inside(l[2], l[1]);
        R side3 = fraction_inside(l[2], l[3]);
        area += R(0.5) * side2 * side3;
        return area;
    }
    if(inside == 1) {
        while(l[0] >= 0) cycle();
        R side0 = fraction_inside(l[0], l[3]);
        R side1 = fraction_inside(l[0], l[1]);
        return R(0.5) * side0 * side1;
    }
    return R(0);
}

template<class R> class FlipOracle {
public:
    orc_params P;
    int G[3];
    R dx, bmin[3], bmax[3], boxMin[3], boxMax[3], sdfRadius, frameDuration, frameTime = 0;
    std::vector<V3<R>> pos, vel;
    std::vector<R> Cmat; // APIC/AFLIP affine matrices, 9 per particle (C[d] row = gradient of component d)
    std::vector<uint32_t> pid;
    Arr3<R> u[3], tmp[3], old[3], dV[3];
    Arr3<char> valid[3], oldValid[3];
    Arr3<R> phi;
    Arr3<uint32_t> activeIdx;
    std::vector<R> rhs, pressure;
    uint32_t nActive = 0, zeroPhiCells = 0;
    uint64_t substepIndex = 0;  // sub-steps taken (keys the position-correction jitter)
    // boundary objects beyond the domain box: [domain box, static..., dynamic...]
    std::vector<OObj<R>> objs;
    int nStatic = 0;
    bool gridBoundary = false;  // a dynamic object: boundary SDF, weights, constraint
    Arr3<R> nodeSdf, weight[3];
    Arr3<char> extrap[3];       // PIC_Data extrapolates: faces the last extrapolation filled
    // last solve
    PCGResult lastSolve;

    explicit FlipOracle(const orc_params& p) : P(p) {
        dx = (R)P.cell_size;
        R pad = dx * (R)P.n_expand_cells;                 // ParticleSolverData.cpp:252-253
        for(int d = 0; d < 3; ++d) {
            boxMin[d] = (R)P.box_min[d]; boxMax[d] = (R)P.box_max[d];
            bmin[d] = boxMin[d] - pad; bmax[d] = boxMax[d] + pad;
            G[d] = (int)(uint32_t)std::ceil((bmax[d] - bmin[d]) / dx);   // Grid.cpp:47
        }
        sdfRadius = dx * R(1.01 * std::sqrt(3.0) / 2.0);  // PIC_Data.cpp:43
        frameDuration = (R)P.frame_duration;
        frameTime = frameDuration;                          // so that the first step starts a frame
        for(int d = 0; d < 3; ++d) {
            int e[3] = {0, 0, 0}; e[d] = 1;
            u[d].resize(G[0] + e[0], G[1] + e[1], G[2] + e[2], 0);
            tmp[d] = u[d]; old[d] = u[d]; dV[d] = u[d];
            valid[d].resize(G[0] + e[0], G[1] + e[1], G[2] + e[2], 0);
            oldValid[d] = valid[d];
        }
        phi.resize(G[0], G[1], G[2], 0);
        activeIdx.resize(G[0], G[1], G[2], 0);
    }

    int nthreads() const { return P.nthreads > 1 ? P.nthreads : 1; }

    // Grid::getGridCoordinate (Grid.h:197): (p - bMin) / cellSize per component
    inline void gridCoord(const V3<R>& p, R g[3]) const {
        g[0] = (p.x - bmin[0]) / dx; g[1] = (p.y - bmin[1]) / dx; g[2] = (p.z - bmin[2]) / dx;
    }

    // ArrayHelpers::interpolateValueLinear 3D (ArrayHelpers.cpp:91-102)
    static R interp(const R pt[3], const Arr3<R>& a) {
        int i, j, k; R fi, fj, fk;
        get_barycentric(pt[0], i, fi, 0, a.sx);
        get_barycentric(pt[1], j, fj, 0, a.sy);
        get_barycentric(pt[2], k, fk, 0, a.sz);
        return trilerp(a(i, j, k), a(i + 1, j, k), a(i, j + 1, k), a(i + 1, j + 1, k),
                       a(i, j, k + 1), a(i + 1, j, k + 1), a(i, j + 1, k + 1), a(i + 1, j + 1, k + 1), fi, fj, fk);
    }
    // PIC_Solver::getVelocityFromGrid (PIC_Solver.cpp:1119-1133)
    R velFromGrid(const R g[3], int d, const Arr3<R>* arr) const {
        R pt[3];
        for(int a = 0; a < 3; ++a) pt[a] = g[a] - (a == d ? R(0) : R(0.5));
        return interp(pt, arr[d]);
    }

    // PIC_Solver::trace_rk2 (PIC_Solver.cpp:1137-1144)
    V3<R> traceRK2(const V3<R>& p, R dt) const {
        R g[3]; gridCoord(p, g);
        V3<R> v{velFromGrid(g, 0, u), velFromGrid(g, 1, u), velFromGrid(g, 2, u)};
        R h = R(0.5) * dt;
        V3<R> mid{p.x + h * v.x, p.y + h * v.y, p.z + h * v.z};
        gridCoord(mid, g);
        v = V3<R>{velFromGrid(g, 0, u), velFromGrid(g, 1, u), velFromGrid(g, 2, u)};
        return V3<R>{p.x + dt * v.x, p.y + dt * v.y, p.z + dt * v.z};
    }

    // BoxObject::signedDistance with bNegativeInside = false (GeometryObjects.cpp:246-268,
    // BoundaryObject.h:47): positive inside the domain box, negative outside.
    R boxSDF(R px, R py, R pz) const {
        R p[3] = {px, py, pz};
        bool inside = true;
        for(int d = 0; d < 3; ++d) if(p[d] < boxMin[d] || p[d] > boxMax[d]) inside = false;
        R mind = std::numeric_limits<R>::max();
        if(inside) {
            for(int d = 0; d < 3; ++d) mind = smin(mind, smin(p[d] - boxMin[d], boxMax[d] - p[d]));
            mind = -mind;
        } else {
            R c[3];
            for(int d = 0; d < 3; ++d) c[d] = smax(smin(p[d], boxMax[d]), boxMin[d]);
            mind = std::sqrt(length2(p[0] - c[0], p[1] - c[1], p[2] - c[2]));
        }
        mind = -mind;
        return R(1.0) * mind;
    }
    // GeometryObject::gradSignedDistance 3D (GeometryObjects.cpp:37-85), dx = 1e-4
    void gradBoxSDF(const V3<R>& p, R g[3]) const {
        const R e = R(1e-4);
        R v000 = boxSDF(p.x - e, p.y - e, p.z - e), v001 = boxSDF(p.x - e, p.y - e, p.z + e);
        R v010 = boxSDF(p.x - e, p.y + e, p.z - e), v011 = boxSDF(p.x - e, p.y + e, p.z + e);
        R v100 = boxSDF(p.x + e, p.y - e, p.z - e), v101 = boxSDF(p.x + e, p.y - e, p.z + e);
        R v110 = boxSDF(p.x + e, p.y + e, p.z - e), v111 = boxSDF(p.x + e, p.y + e, p.z + e);
        R ddx00 = v100 - v000, ddx10 = v110 - v010, ddx01 = v101 - v001, ddx11 = v111 - v011;
        R ddy00 = v010 - v000, ddy10 = v110 - v100, ddy01 = v011 - v001, ddy11 = v111 - v101;
        R ddz00 = v001 - v000, ddz10 = v101 - v100, ddz01 = v011 - v010, ddz11 = v111 - v110;
        g[0] = (((ddx00 + ddx01) + ddx10) + ddx11) * R(0.25);
        g[1] = (((ddy00 + ddy01) + ddy10) + ddy11) * R(0.25);
        g[2] = (((ddz00 + ddz01) + ddz10) + ddz11) * R(0.25);
    }
    // GeometryObject::invTransform + Box / SphereObject::signedDistance(p, false)
    // (GeometryObjects.cpp:231-268,379-384): positive inside the object
    static R objSDF(const OObj<R>& o, R x, R y, R z) {
        R q[3] = {x, y, z};
        if(o.transformed)
            for(int r = 0; r < 3; ++r) q[r] = ((o.M[4 * r] * x + o.M[4 * r + 1] * y) + o.M[4 * r + 2] * z) + o.M[4 * r + 3];
        if(o.geometry == 0) {
            bool inside = true;
            for(int d = 0; d < 3; ++d) if(q[d] < o.bmin[d] || q[d] > o.bmax[d]) inside = false;
            R mind = std::numeric_limits<R>::max();
            if(inside) {
                for(int d = 0; d < 3; ++d) mind = smin(mind, smin(q[d] - o.bmin[d], o.bmax[d] - q[d]));
                mind = -mind;
            } else {
                R c[3];
                for(int d = 0; d < 3; ++d) c[d] = smax(smin(q[d], o.bmax[d]), o.bmin[d]);
                mind = std::sqrt(length2(q[0] - c[0], q[1] - c[1], q[2] - c[2]));
            }
            mind = -mind;
            return o.scale * mind;
        }
        R d = o.scale * (std::sqrt(length2(q[0], q[1], q[2])) - R(1.0));
        return -d;
    }
    // boundary group grp: 0 = CSG union of the static objects (CSGObject::signedDistance,
    // GeometryObjects.cpp:861-896), g > 0 = the g-th dynamic object
    R groupSDF(int grp, R x, R y, R z) const {
        int b = grp == 0 ? 0 : nStatic + grp - 1, e = grp == 0 ? nStatic : b + 1;
        R sd = objSDF(objs[b], x, y, z);
        for(int i = b + 1; i < e; ++i) sd = smin(sd, objSDF(objs[i], x, y, z));
        return sd;
    }
    int nGroups() const { return objs.empty() ? 0 : 1 + (int)objs.size() - nStatic; }

    // BoundaryObject::constrainToBoundary(ppos, pvel) (BoundaryObject.cpp:72-90), no
    // reflection, for every boundary object in turn (PIC_Solver.cpp:353-372)
    void constrain(V3<R>& p) const {
        if(!objs.empty()) {
            for(int grp = 0; grp < nGroups(); ++grp) {
                R phiVal = groupSDF(grp, p.x, p.y, p.z);
                if(!(phiVal < 0)) continue;
                const R e = R(1e-4);
                R v000 = groupSDF(grp, p.x - e, p.y - e, p.z - e), v001 = groupSDF(grp, p.x - e, p.y - e, p.z + e);
                R v010 = groupSDF(grp, p.x - e, p.y + e, p.z - e), v011 = groupSDF(grp, p.x - e, p.y + e, p.z + e);
                R v100 = groupSDF(grp, p.x + e, p.y - e, p.z - e), v101 = groupSDF(grp, p.x + e, p.y - e, p.z + e);
                R v110 = groupSDF(grp, p.x + e, p.y + e, p.z - e), v111 = groupSDF(grp, p.x + e, p.y + e, p.z + e);
                R g[3];
                g[0] = ((((v100 - v000) + (v101 - v001)) + (v110 - v010)) + (v111 - v011)) * R(0.25);
                g[1] = ((((v010 - v000) + (v011 - v001)) + (v110 - v100)) + (v111 - v101)) * R(0.25);
                g[2] = ((((v001 - v000) + (v011 - v010)) + (v101 - v100)) + (v111 - v110)) * R(0.25);
                R m2 = length2(g[0], g[1], g[2]);
                if(m2 > std::numeric_limits<R>::min()) {
                    R sq = std::sqrt(m2);
                    g[0] /= sq; g[1] /= sq; g[2] /= sq;
                    p.x -= phiVal * g[0]; p.y -= phiVal * g[1]; p.z -= phiVal * g[2];
                }
            }
            return;
        }
        R phiVal = boxSDF(p.x, p.y, p.z);
        if(phiVal < 0) {
            R g[3]; gradBoxSDF(p, g);
            R m2 = length2(g[0], g[1], g[2]);
            if(m2 > std::numeric_limits<R>::min()) {
                R s = std::sqrt(m2);
                g[0] /= s; g[1] /= s; g[2] /= s;
                p.x -= phiVal * g[0]; p.y -= phiVal * g[1]; p.z -= phiVal * g[2];
            }
        }
    }

    // ParticleSolver::generateBoundaries (ParticleSolver.cpp:242-295) + computeBoundarySDF
    // (PIC_Solver.cpp:1157-1168) + computeCellWeights (PIC_Solver.cpp:543-598)
    void setBoundaries(const orc_boundary_object* in, uint32_t n, bool updateGrid) {
        objs.clear();
        nStatic = 0;
        if(n == 0) { gridBoundary = false; return; }
        bool anyDynamic = false;
        OObj<R> box;
        for(int d = 0; d < 3; ++d) { box.bmin[d] = boxMin[d]; box.bmax[d] = boxMax[d]; }
        objs.push_back(box);
        for(int pass = 0; pass < 2; ++pass)
            for(uint32_t i = 0; i < n; ++i) {
                if((in[i].dynamic != 0) != (pass == 1)) continue;
                OObj<R> o;
                o.geometry = in[i].geometry;
                o.transformed = in[i].transformed ? 1 : 0;
                o.scale = (R)in[i].uniform_scale;
                for(int d = 0; d < 3; ++d) { o.bmin[d] = (R)in[i].box_min[d]; o.bmax[d] = (R)in[i].box_max[d]; }
                for(int q = 0; q < 12; ++q) o.M[q] = (R)in[i].inv_transform[q];
                objs.push_back(o);
                if(pass == 1) anyDynamic = true;
            }
        nStatic = 1;
        for(uint32_t i = 0; i < n; ++i) nStatic += in[i].dynamic ? 0 : 1;
        if(!(anyDynamic && updateGrid)) return;
        gridBoundary = true;
        nodeSdf.resize(G[0] + 1, G[1] + 1, G[2] + 1, 0);
        for(int k = 0; k <= G[2]; ++k)
            for(int j = 0; j <= G[1]; ++j)
                for(int i = 0; i <= G[0]; ++i) {
                    R x = bmin[0] + (R)i * dx, y = bmin[1] + (R)j * dx, z = bmin[2] + (R)k * dx;
                    R m = std::numeric_limits<R>::max();
                    for(int grp = 0; grp < nGroups(); ++grp) m = smin(m, groupSDF(grp, x, y, z));
                    nodeSdf(i, j, k) = m;
                }
        for(int d = 0; d < 3; ++d) {
            weight[d].resize(u[d].sx, u[d].sy, u[d].sz, 0);
            for(int k = 0; k < u[d].sz; ++k)
                for(int j = 0; j < u[d].sy; ++j)
                    for(int i = 0; i < u[d].sx; ++i) {
                        const Arr3<R>& N = nodeSdf;
                        R f;
                        if(d == 0) f = fraction_inside4(N(i, j, k), N(i, j + 1, k), N(i, j, k + 1), N(i, j + 1, k + 1));
                        else if(d == 1) f = fraction_inside4(N(i, j, k), N(i, j, k + 1), N(i + 1, j, k), N(i + 1, j, k + 1));
                        else f = fraction_inside4(N(i, j, k), N(i, j + 1, k), N(i + 1, j, k), N(i + 1, j + 1, k));
                        R t = R(1.0) - f;
                        weight[d](i, j, k) = t < 0 ? R(0) : (t > R(1.0) ? R(1.0) : t);
                    }
        }
    }
    R faceWeight(int d, int i, int j, int k) const { return gridBoundary ? weight[d](i, j, k) : R(1.0); }

    // ArrayHelpers::interpolateGradient 3D (ArrayHelpers.cpp:214-251)
    static void interpGradient(const R pt[3], const Arr3<R>& a, R out[3]) {
        int i, j, k; R fi, fj, fk;
        get_barycentric(pt[0], i, fi, 0, a.sx);
        get_barycentric(pt[1], j, fj, 0, a.sy);
        get_barycentric(pt[2], k, fk, 0, a.sz);
        R v000 = a(i, j, k), v001 = a(i, j, k + 1), v010 = a(i, j + 1, k), v011 = a(i, j + 1, k + 1);
        R v100 = a(i + 1, j, k), v101 = a(i + 1, j, k + 1), v110 = a(i + 1, j + 1, k), v111 = a(i + 1, j + 1, k + 1);
        out[0] = bilerp(v100 - v000, v110 - v010, v101 - v001, v111 - v011, fj, fk);
        out[1] = bilerp(v010 - v000, v110 - v100, v011 - v001, v111 - v101, fi, fk);
        out[2] = bilerp(v001 - v000, v101 - v100, v011 - v010, v111 - v110, fi, fj);
    }

    // PIC_Solver::constrainGridVelocity (PIC_Solver.cpp:1093-1115)
    void constrainGridVelocity() {
        for(int d = 0; d < 3; ++d) {
            tmp[d].d = u[d].d;
            for(int k = 0; k < u[d].sz; ++k)
                for(int j = 0; j < u[d].sy; ++j)
                    for(int i = 0; i < u[d].sx; ++i) {
                        if(!(extrap[d](i, j, k) == 1 && weight[d](i, j, k) < std::numeric_limits<R>::min())) continue;
                        R gp[3] = {(R)i + (d == 0 ? R(0) : R(0.5)), (R)j + (d == 1 ? R(0) : R(0.5)),
                                   (R)k + (d == 2 ? R(0) : R(0.5))};
                        R vel[3] = {velFromGrid(gp, 0, u), velFromGrid(gp, 1, u), velFromGrid(gp, 2, u)};
                        R nrm[3];
                        interpGradient(gp, nodeSdf, nrm);
                        R m2 = length2(nrm[0], nrm[1], nrm[2]);
                        if(m2 > std::numeric_limits<R>::min()) {
                            R sq = std::sqrt(m2);
                            nrm[0] /= sq; nrm[1] /= sq; nrm[2] /= sq;
                            R dn = (vel[0] * nrm[0] + vel[1] * nrm[1]) + vel[2] * nrm[2];
                            tmp[d](i, j, k) = vel[d] - dn * nrm[d];
                        }
                    }
            u[d].d = tmp[d].d;
        }
    }

    // PIC_Solver::timestepCFL (PIC_Solver.cpp:342-349)
    R timestepCFL() const {
        R maxVel = std::numeric_limits<R>::min();
        for(int d = 0; d < 3; ++d) maxVel = smax(maxVel, max_abs(u[d].d.data(), u[d].size()));
        R ts = maxVel > std::numeric_limits<R>::min() ? (R)P.cfl_factor * (dx / maxVel) : std::numeric_limits<R>::max();
        R lo = (R)P.min_timestep, hi = (R)P.max_timestep;
        return ts < lo ? lo : (ts > hi ? hi : ts);
    }

    // PIC_Solver::moveParticles (PIC_Solver.cpp:353-373)
    void moveParticles(R dt) {
        R sub = dt / R(P.advection_steps);
#pragma omp parallel for schedule(static) if(nthreads() > 1)
        for(long long p = 0; p < (long long)pos.size(); ++p) {
            V3<R> pp = pos[p];
            for(uint32_t i = 0; i < P.advection_steps; ++i) {
                pp = traceRK2(pp, sub);
                constrain(pp);
            }
            pos[p] = pp;
        }
    }

    // Counter-based jitter replacing NumberHelpers::fRand11::vrnd (a process-global MT
    // stream, NumberHelpers.h:155-258): three values in [-1, 1) from SplitMix64 over
    // (sub-step, particle id, neighbour id), 21 bits each.
    static uint64_t smix(uint64_t x) {
        x += 0x9E3779B97F4A7C15ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    }
    static void jitter(uint64_t step, uint32_t a, uint32_t b, R out[3]) {
        const uint64_t h = smix(smix(smix(step) ^ (uint64_t)a) ^ (uint64_t)b);
        for(int c = 0; c < 3; ++c) {
            const float u = (float)((h >> (21 * c)) & 0x1FFFFFull) * (1.0f / 2097152.0f);
            out[c] = (R)(2.0f * u - 1.0f);
        }
    }
    // MathHelpers::smooth_kernel (MathHelpers.h:661-664): (1 - r2/h2)^3 inside h.  The cube
    // is the rounding of the double product, the same on every platform (pow's last bit is
    // implementation-defined).
    static R smoothKernel(R r2, R h2) {
        const R x2 = r2 / h2;
        if(x2 > R(1.0)) return R(0);
        const R t = R(1.0) - x2;
        return (R)(((double)t * (double)t) * (double)t);
    }

    // PIC_Solver::correctParticlePositions (PIC_Solver.cpp:377-485), 3D: each particle is
    // pushed by springs to the other particles of its 3x3x3 cells (cells z, y, x major, the
    // particles of a cell in id order), jittered where two nearly coincide, then moved and
    // projected into the box AdvectionSteps times; all particles read the old positions.
    // Needs the particles sorted by (cell, id).
    void correctPositions(R timestep) {
        const size_t n = pos.size(), C = (size_t)G[0] * G[1] * G[2];
        std::vector<uint32_t> start(C + 1, 0);
        for(size_t p = 0; p < n; ++p) start[cellLinear(pos[p]) + 1]++;
        for(size_t c = 0; c < C; ++c) start[c + 1] += start[c];
        const R particleRadius = R(P.cell_size) / R(P.ratio_cell_size_p_radius);
        const R radius = R(2.0) * particleRadius / R(std::sqrt(3.0));
        const R radius2 = radius * radius;
        const R threshold = R(0.01) * radius;
        const R threshold2 = threshold * threshold;
        const R substep = timestep / R(P.advection_steps);
        const R kSpring = radius * substep * R(P.repulsive_force_stiffness);
        std::vector<V3<R>> out(n);
#pragma omp parallel for schedule(static) if(nthreads() > 1)
        for(long long p = 0; p < (long long)n; ++p) {
            const V3<R> pp = pos[p];
            int c[3];
            cellOf(pp, c);
            R spring[3] = {R(0), R(0), R(0)};
            for(int dk = -1; dk <= 1; ++dk)
                for(int dj = -1; dj <= 1; ++dj)
                    for(int di = -1; di <= 1; ++di) {
                        const int ci = c[0] + di, cj = c[1] + dj, ck = c[2] + dk;
                        if(ci < 0 || cj < 0 || ck < 0 || ci >= G[0] || cj >= G[1] || ck >= G[2]) continue;
                        const size_t cell = ((size_t)ck * G[1] + cj) * G[0] + ci;
                        for(uint32_t q = start[cell]; q < start[cell + 1]; ++q) {
                            if((long long)q == p) continue;
                            const R x[3] = {pp.x - pos[q].x, pp.y - pos[q].y, pp.z - pos[q].z};
                            const R d2 = length2(x[0], x[1], x[2]);
                            const R w = smoothKernel(d2, radius2);
                            if(d2 > threshold2) {
                                const R s = std::sqrt(d2);
                                for(int a = 0; a < 3; ++a) spring[a] += w * x[a] / s;
                            } else {
                                R j[3];
                                jitter(substepIndex, pid[p], pid[q], j);
                                const R f = threshold / timestep;
                                for(int a = 0; a < 3; ++a) spring[a] += f * j[a];
                            }
                        }
                    }
            V3<R> np = pp;
            for(uint32_t s = 0; s < P.advection_steps; ++s) {
                np.x += spring[0] * kSpring;
                np.y += spring[1] * kSpring;
                np.z += spring[2] * kSpring;
                constrain(np);
            }
            out[p] = np;
        }
        pos.swap(out);
    }

    // Grid::getCellIdx<Int> (Grid.h:156-162) clamped into the grid, linearised (Grid.h:108-111)
    inline void cellOf(const V3<R>& p, int c[3]) const {
        c[0] = (int)((p.x - bmin[0]) / dx); c[1] = (int)((p.y - bmin[1]) / dx); c[2] = (int)((p.z - bmin[2]) / dx);
    }
    inline uint32_t cellLinear(const V3<R>& p) const {
        int c[3]; cellOf(p, c);
        for(int d = 0; d < 3; ++d) c[d] = c[d] < 0 ? 0 : (c[d] > G[d] - 1 ? G[d] - 1 : c[d]);
        return (uint32_t)(((size_t)c[2] * G[1] + c[1]) * G[0] + c[0]);
    }

    // Grid::collectIndexToCells (one thread, so each bucket lists particles in index
    // order) + getParticleIdxSortedByCell + sortData (Grid.cpp:92-114,283-309), applied to
    // the particles in their original (id) order: the result is sorted by (cell, id)
    // whatever order the particles are stored in.
    void sortParticlesByCell() {
        size_t n = pos.size(), C = (size_t)G[0] * G[1] * G[2];
        std::vector<uint32_t> key(n), start(C + 1, 0), order(n), byId(n);
        for(size_t p = 0; p < n; ++p) byId[pid[p]] = (uint32_t)p;
        for(size_t p = 0; p < n; ++p) { key[p] = cellLinear(pos[p]); start[key[p] + 1]++; }
        for(size_t c = 0; c < C; ++c) start[c + 1] += start[c];
        for(size_t q = 0; q < n; ++q) { uint32_t p = byId[q]; order[start[key[p]]++] = p; }
        std::vector<V3<R>> np(n), nv(n);
        std::vector<uint32_t> ni(n);
        std::vector<R> nc(Cmat.size());
        for(size_t i = 0; i < n; ++i) {
            np[i] = pos[order[i]]; nv[i] = vel[order[i]]; ni[i] = pid[order[i]];
            if(!Cmat.empty()) for(int q = 0; q < 9; ++q) nc[i * 9 + q] = Cmat[(size_t)order[i] * 9 + q];
        }
        pos.swap(np); vel.swap(nv); pid.swap(ni); Cmat.swap(nc);
    }

    // ArrayHelpers::getCoordinatesAndWeights 3D (ArrayHelpers.cpp:50-76)
    static void coordsWeights(const R pt[3], const Arr3<R>& a, int idx[8][3], R w[8]) {
        int i, j, k; R fi, fj, fk;
        get_barycentric(pt[0], i, fi, 0, a.sx);
        get_barycentric(pt[1], j, fj, 0, a.sy);
        get_barycentric(pt[2], k, fk, 0, a.sz);
        int c[8][3] = {{i, j, k}, {i + 1, j, k}, {i, j + 1, k}, {i + 1, j + 1, k},
                       {i, j, k + 1}, {i + 1, j, k + 1}, {i, j + 1, k + 1}, {i + 1, j + 1, k + 1}};
        std::memcpy(idx, c, sizeof(c));
        w[0] = (R(1.0) - fi) * (R(1.0) - fj) * (R(1.0) - fk);
        w[1] = fi * (R(1.0) - fj) * (R(1.0) - fk);
        w[2] = (R(1.0) - fi) * fj * (R(1.0) - fk);
        w[3] = fi * fj * (R(1.0) - fk);
        w[4] = (R(1.0) - fi) * (R(1.0) - fj) * fk;
        w[5] = fi * (R(1.0) - fj) * fk;
        w[6] = (R(1.0) - fi) * fj * fk;
        w[7] = fi * fj * fk;
    }

    // P2G with the sums in the canonical two-level order of the CUDA kernel: for every
    // face, the particles of each candidate cell (two along the component's own axis, three
    // along the others, clamped to the grid) are summed in id order into a per-cell
    // partial, and the face adds its candidate cells' partials in (y, z, x)-major cell
    // order, both sums starting at +0.  The products are those of mapP2G
    // (getCoordinatesAndWeights, ArrayHelpers.cpp:50-76, weight = wx * wy * wz left to
    // right, momentum = weight * v, and for APIC / AFLIP weight * (v + C_d . (x_face - x_p))
    // with the face's world position, APIC_Solver.cpp:53-91); only the association of the
    // sums differs from the reference's serial loop, whose CAS-atomic parallel form
    // (FLIP_Solver.cpp:57-95, AtomicOperations.h:31-49) has no fixed order.  Needs the
    // particles sorted by (cell, id).  Faces are independent, so this runs on any number of
    // threads with the same result.
    void mapP2GCanonical() {
        const bool affine = (P.solver_kind == 1 || P.solver_kind == 2);
        const size_t n = pos.size(), C = (size_t)G[0] * G[1] * G[2];
        std::vector<uint32_t> start(C + 1, 0);
        for(size_t p = 0; p < n; ++p) start[cellLinear(pos[p]) + 1]++;
        for(size_t c = 0; c < C; ++c) start[c + 1] += start[c];
        // stencil base index and fraction of every particle, component and axis
        std::vector<int> base(n * 9);
        std::vector<R> frac(n * 9);
#pragma omp parallel for schedule(static) if(nthreads() > 1)
        for(long long p = 0; p < (long long)n; ++p) {
            R g[3];
            gridCoord(pos[p], g);
            for(int d = 0; d < 3; ++d)
                for(int a = 0; a < 3; ++a) {
                    const int size = G[a] + (a == d ? 1 : 0);
                    int i; R f;
                    get_barycentric(g[a] - (a == d ? R(0) : R(0.5)), i, f, 0, size);
                    base[(size_t)p * 9 + d * 3 + a] = i;
                    frac[(size_t)p * 9 + d * 3 + a] = f;
                }
        }
        for(int d = 0; d < 3; ++d) {
            Arr3<R>& out = u[d];
            Arr3<R>& wsum = tmp[d];
            std::fill(valid[d].d.begin(), valid[d].d.end(), 0);
            const int sx = out.sx, sy = out.sy, sz = out.sz;
#pragma omp parallel for schedule(static) if(nthreads() > 1)
            for(long long li = 0; li < (long long)out.size(); ++li) {
                const int f[3] = {(int)(li % sx), (int)((li / sx) % sy), (int)(li / ((long long)sx * sy))};
                int lo[3], hi[3];
                for(int a = 0; a < 3; ++a) {
                    lo[a] = std::max(f[a] - 1, 0);
                    hi[a] = std::min(a == d ? f[a] : f[a] + 1, G[a] - 1);
                }
                R S = R(0), W = R(0);
                for(int cy = lo[1]; cy <= hi[1]; ++cy)
                    for(int cz = lo[2]; cz <= hi[2]; ++cz)
                        for(int cx = lo[0]; cx <= hi[0]; ++cx) {
                            const size_t c = ((size_t)cz * G[1] + cy) * G[0] + cx;
                            R PS = R(0), PW = R(0);
                            for(uint32_t q = start[c]; q < start[c + 1]; ++q) {
                                const int* b = &base[(size_t)q * 9 + d * 3];
                                const R* fr = &frac[(size_t)q * 9 + d * 3];
                                R w3[3];
                                bool reach = true;
                                for(int a = 0; a < 3; ++a) {
                                    if(f[a] == b[a]) w3[a] = R(1.0) - fr[a];
                                    else if(f[a] == b[a] + 1) w3[a] = fr[a];
                                    else reach = false;
                                }
                                if(!reach) continue;
                                const R w = w3[0] * w3[1] * w3[2];
                                R m;
                                if(affine) {
                                    // gpos = grid().getWorldCoordinate(VecN(face) + extra) (Grid.h:181-184)
                                    R gp[3];
                                    for(int a = 0; a < 3; ++a) gp[a] = ((R)f[a] + (a == d ? R(0) : R(0.5))) * dx + bmin[a];
                                    const R* Cq = &Cmat[(size_t)q * 9 + d * 3];
                                    const R dxp = gp[0] - pos[q].x, dyp = gp[1] - pos[q].y, dzp = gp[2] - pos[q].z;
                                    const R dotv = (Cq[0] * dxp + Cq[1] * dyp) + Cq[2] * dzp;
                                    m = w * (vel[q][d] + dotv);
                                } else {
                                    m = w * vel[q][d];
                                }
                                PS = PS + m;
                                PW = PW + w;
                            }
                            S = S + PS;
                            W = W + PW;
                        }
                out.d[li] = S;
                wsum.d[li] = W;
            }
#pragma omp parallel for schedule(static) if(nthreads() > 1)
            for(long long i = 0; i < (long long)out.size(); ++i) {
                R w = wsum.d[i];
                if(w > std::numeric_limits<R>::min()) { out.d[i] /= w; valid[d].d[i] = 1; }
            }
        }
    }

    // Which P2G the step runs: FLIP, APIC and AFLIP in the canonical mode take the
    // two-level order above; every other case the reference's serial loop.
    void splatParticles() {
        if(P.solver_kind <= 2 && P.reduce_mode == 1 && (P.sort_each_step || P.correct_position)) mapP2GCanonical();
        else mapP2G();
    }

    // FLIP_Solver::mapParticles2Grid (FLIP_Solver.cpp:57-95); APIC adds the affine term
    // (APIC_Solver.cpp:53-91).  Serial in particle-array order.
    void mapP2G() {
        for(int d = 0; d < 3; ++d) {
            std::fill(u[d].d.begin(), u[d].d.end(), R(0));
            std::fill(tmp[d].d.begin(), tmp[d].d.end(), R(0));
            std::fill(valid[d].d.begin(), valid[d].d.end(), 0);
        }
        bool affine = (P.solver_kind == 1 || P.solver_kind == 2);
        auto splat = [&](size_t p) {
            R g[3]; gridCoord(pos[p], g);
            for(int d = 0; d < 3; ++d) {
                R pt[3]; for(int a = 0; a < 3; ++a) pt[a] = g[a] - (a == d ? R(0) : R(0.5));
                int idx[8][3]; R w[8];
                coordsWeights(pt, u[d], idx, w);
                for(int n = 0; n < 8; ++n) {
                    R m;
                    if(affine) {
                        // gpos = grid().getWorldCoordinate(VecN(indices[i]) + extra) (Grid.h:181-184)
                        R gp[3];
                        for(int a = 0; a < 3; ++a) gp[a] = ((R)idx[n][a] + (a == d ? R(0) : R(0.5))) * dx + bmin[a];
                        const R* C = &Cmat[p * 9 + d * 3];
                        R dxp = gp[0] - pos[p].x, dyp = gp[1] - pos[p].y, dzp = gp[2] - pos[p].z;
                        R dotv = (C[0] * dxp + C[1] * dyp) + C[2] * dzp;
                        m = w[n] * (vel[p][d] + dotv);
                    } else {
                        m = w[n] * vel[p][d];
                    }
                    size_t li = u[d].lin(idx[n][0], idx[n][1], idx[n][2]);
                    if(nthreads() > 1) {
                        std::atomic_ref<R>(u[d].d[li]).fetch_add(m);
                        std::atomic_ref<R>(tmp[d].d[li]).fetch_add(w[n]);
                    } else {
                        u[d].d[li] = u[d].d[li] + m;
                        tmp[d].d[li] = tmp[d].d[li] + w[n];
                    }
                }
            }
        };
        if(nthreads() > 1) {
#pragma omp parallel for schedule(static)
            for(long long p = 0; p < (long long)pos.size(); ++p) splat((size_t)p);
        } else {
            for(size_t p = 0; p < pos.size(); ++p) splat(p);
        }
        for(int d = 0; d < 3; ++d) {
#pragma omp parallel for schedule(static) if(nthreads() > 1)
            for(long long i = 0; i < (long long)u[d].size(); ++i) {
                R w = tmp[d].d[i];
                if(w > std::numeric_limits<R>::min()) { u[d].d[i] /= w; valid[d].d[i] = 1; }
            }
        }
    }

    // PIC_Solver::extrapolateVelocity (PIC_Solver.cpp:985-1090); `ext` marks the faces this
    // call filled (the extrapolates flags constrainGridVelocity reads)
    void extrapolate(Arr3<R>& grid, Arr3<R>& temp, Arr3<char>& vld, Arr3<char>& ovld, Arr3<char>& ext) {
        ext.resize(grid.sx, grid.sy, grid.sz, 0);
        temp.d = grid.d;
        for(int layer = 0; layer < 4; ++layer) {
            ovld.d = vld.d;
#pragma omp parallel for schedule(static) if(nthreads() > 1)
            for(int k = 1; k < grid.sz - 1; ++k)
                for(int j = 1; j < grid.sy - 1; ++j)
                    for(int i = 1; i < grid.sx - 1; ++i) {
                        if(ovld(i, j, k)) continue;
                        R sum = 0; uint32_t count = 0;
                        if(ovld(i + 1, j, k)) { sum += grid(i + 1, j, k); ++count; }
                        if(ovld(i - 1, j, k)) { sum += grid(i - 1, j, k); ++count; }
                        if(ovld(i, j + 1, k)) { sum += grid(i, j + 1, k); ++count; }
                        if(ovld(i, j - 1, k)) { sum += grid(i, j - 1, k); ++count; }
                        if(ovld(i, j, k + 1)) { sum += grid(i, j, k + 1); ++count; }
                        if(ovld(i, j, k - 1)) { sum += grid(i, j, k - 1); ++count; }
                        if(count > 0) { temp(i, j, k) = sum / static_cast<R>(count); vld(i, j, k) = 1; ext(i, j, k) = 1; }
                    }
            grid.d = temp.d;
        }
    }
    void extrapolateAll() { for(int d = 0; d < 3; ++d) extrapolate(u[d], tmp[d], valid[d], oldValid[d], extrap[d]); }

    // PIC_Solver::advectGridVelocity + trace_rk2_grid (PIC_Solver.cpp:489-501, 1148-1154):
    // semi-Lagrangian back-trace of every face through the grid velocity, RK2 in grid
    // units (velocity x invCellSize, Grid.cpp:38-44).  Each component is copied back before
    // the next one is advected, so v is traced through the advected u, and w through both.
    void advectGrid(R dt) {
        const R inv = R(1.0) / dx;
        const R ts = -dt;
        for(int d = 0; d < 3; ++d) {
            Arr3<R>& out = tmp[d];
            const int sx = u[d].sx, sy = u[d].sy, sz = u[d].sz;
#pragma omp parallel for schedule(static) if(nthreads() > 1)
            for(int k = 0; k < sz; ++k)
                for(int j = 0; j < sy; ++j)
                    for(int i = 0; i < sx; ++i) {
                        const R gp[3] = {(R)i + (d == 0 ? R(0) : R(0.5)), (R)j + (d == 1 ? R(0) : R(0.5)),
                                         (R)k + (d == 2 ? R(0) : R(0.5))};
                        R gv[3];
                        for(int c = 0; c < 3; ++c) gv[c] = velFromGrid(gp, c, u) * inv;
                        const R h = R(0.5) * ts;
                        R mid[3];
                        for(int c = 0; c < 3; ++c) mid[c] = gp[c] + h * gv[c];
                        for(int c = 0; c < 3; ++c) gv[c] = velFromGrid(mid, c, u) * inv;
                        R back[3];
                        for(int c = 0; c < 3; ++c) back[c] = gp[c] + ts * gv[c];
                        out(i, j, k) = velFromGrid(back, d, u);
                    }
            u[d].d = out.d;
        }
    }

    // PIC_Solver::addGravity, Earth gravity (PIC_Solver.cpp:505-511)
    void addGravity(R dt) {
        if(!P.apply_gravity) return;
        R g = R(9.81) * dt;
        for(auto& v : u[1].d) v -= g;
    }

    // PIC_Solver::computeFluidSDF (PIC_Solver.cpp:601-689).  The solid-extension pass
    // only fires where boundarySDF < 0; boundarySDF is never computed for a static scene
    // (computeBoundarySDF is only called for dynamic boundaries, PIC_Solver.cpp:105-114)
    // and stays 0 (PIC_Data.cpp:116), so that pass is a no-op here.
    void computeFluidSDF() {
        std::fill(phi.d.begin(), phi.d.end(), dx * R(3.0));
        auto body = [&](size_t p) {
            const V3<R>& pp = pos[p];
            int c[3]; cellOf(pp, c);
            int lo[3], hi[3];
            for(int a = 0; a < 3; ++a) { lo[a] = std::max(0, c[a] - 1); hi[a] = std::min(c[a] + 1, G[a] - 1); }
            for(int k = lo[2]; k <= hi[2]; ++k)
                for(int j = lo[1]; j <= hi[1]; ++j)
                    for(int i = lo[0]; i <= hi[0]; ++i) {
                        R sx = (R)(i + 0.5) * dx + bmin[0], sy = (R)(j + 0.5) * dx + bmin[1], sz = (R)(k + 0.5) * dx + bmin[2];
                        R val = std::sqrt(length2(sx - pp.x, sy - pp.y, sz - pp.z)) - sdfRadius;
                        R& cur = phi(i, j, k);
                        if(nthreads() > 1) {
                            std::atomic_ref<R> ar(cur);
                            R o = ar.load();
                            while(val < o && !ar.compare_exchange_weak(o, val)) {}
                        } else if(val < cur) {
                            cur = val;
                        }
                    }
        };
        if(nthreads() > 1) {
#pragma omp parallel for schedule(static)
            for(long long p = 0; p < (long long)pos.size(); ++p) body((size_t)p);
        } else {
            for(size_t p = 0; p < pos.size(); ++p) body(p);
        }
        if(!gridBoundary) return;
        // solid part (PIC_Solver.cpp:671-688)
        const R half = R(0.5) * dx;
        for(int k = 0; k < G[2]; ++k)
            for(int j = 0; j < G[1]; ++j)
                for(int i = 0; i < G[0]; ++i) {
                    if(!(phi(i, j, k) < half)) continue;
                    const Arr3<R>& N = nodeSdf;
                    R solid = R(0.125) * (N(i, j, k) + N(i + 1, j, k) + N(i, j + 1, k) + N(i + 1, j + 1, k) +
                                          N(i, j, k + 1) + N(i + 1, j, k + 1) + N(i, j + 1, k + 1) + N(i + 1, j + 1, k + 1));
                    if(solid < 0) phi(i, j, k) = -half;
                }
    }

    // PIC_Solver::computeSystem (PIC_Solver.cpp:693-893) with static-scene weights = 1.
    // Cells whose fluid SDF is exactly 0 are left out of the system: the reference gives
    // them no active index yet still writes a row for them (at index 0, racing with the
    // real row 0), which has no defined result.
    CSR A;
    std::vector<R> Avals;
    std::vector<float> Adiag; // diagonal per row (0 for rows the loop never writes)
    void computeSystem(R dt) {
        size_t C = phi.size();
        nActive = 0; zeroPhiCells = 0;
        for(size_t i = 0; i < C; ++i) {
            activeIdx.d[i] = 0;
            if(phi.d[i] < 0) activeIdx.d[i] = nActive++;
        }
        rhs.assign(nActive, 0);
        pressure.assign(nActive, 0);
        std::vector<RowBuilder<R>> rows(nActive);
        const Arr3<R>& U = u[0]; const Arr3<R>& V = u[1]; const Arr3<R>& W = u[2];
        const R wgt = R(1.0);
        for(int k = 1; k < G[2] - 1; ++k)
            for(int j = 1; j < G[1] - 1; ++j)
                for(int i = 1; i < G[0] - 1; ++i) {
                    R pc = phi(i, j, k);
                    if(pc > 0) continue;
                    if(!(pc < 0)) { ++zeroPhiCells; continue; }
                    R pr = phi(i + 1, j, k), pl = phi(i - 1, j, k), pt = phi(i, j + 1, k), pb = phi(i, j - 1, k);
                    R pf = phi(i, j, k + 1), pn = phi(i, j, k - 1);
                    R rv = 0;
                    const R wr = gridBoundary ? weight[0](i + 1, j, k) : wgt, wl = gridBoundary ? weight[0](i, j, k) : wgt;
                    const R wt = gridBoundary ? weight[1](i, j + 1, k) : wgt, wb = gridBoundary ? weight[1](i, j, k) : wgt;
                    const R wf = gridBoundary ? weight[2](i, j, k + 1) : wgt, wn = gridBoundary ? weight[2](i, j, k) : wgt;
                    R term_right = wr * dt; rv -= wr * U(i + 1, j, k);
                    R term_left = wl * dt;  rv += wl * U(i, j, k);
                    R term_top = wt * dt;   rv -= wt * V(i, j + 1, k);
                    R term_bottom = wb * dt; rv += wb * V(i, j, k);
                    R term_far = wf * dt;   rv -= wf * W(i, j, k + 1);
                    R term_near = wn * dt;  rv += wn * W(i, j, k);
                    uint32_t c = activeIdx(i, j, k);
                    rhs[c] = rv;
                    R center = 0;
                    RowBuilder<R>& row = rows[c];
                    auto nb = [&](R pn_, R term, int ii, int jj, int kk) {
                        if(pn_ < 0) { center += term; row.add(activeIdx(ii, jj, kk), -term); }
                        else { R th = smax(R(0.01), fraction_inside(pc, pn_)); center += term / th; }
                    };
                    nb(pr, term_right, i + 1, j, k);
                    nb(pl, term_left, i - 1, j, k);
                    nb(pt, term_top, i, j + 1, k);
                    nb(pb, term_bottom, i, j - 1, k);
                    nb(pf, term_far, i, j, k + 1);
                    nb(pn, term_near, i, j, k - 1);
                    row.add(c, center);
                }
        A.n = nActive;
        A.rowStart.assign(nActive + 1, 0);
        for(uint32_t r = 0; r < nActive; ++r) A.rowStart[r + 1] = A.rowStart[r] + rows[r].cnt;
        A.colIndex.resize(A.rowStart[nActive]);
        Avals.resize(A.rowStart[nActive]);
        Adiag.assign(nActive, 0.0f);
        for(uint32_t r = 0; r < nActive; ++r)
            for(int q = 0; q < rows[r].cnt; ++q) {
                A.colIndex[A.rowStart[r] + q] = rows[r].col[q];
                Avals[A.rowStart[r] + q] = rows[r].val[q];
                if(rows[r].col[q] == r) Adiag[r] = (float)rows[r].val[q];
            }
    }

    // PIC_Solver::solveSystem (PIC_Solver.cpp:897-907) -> PCGSolver::solve_precond
    void solveSystem() {
        R tolf = (R)P.cg_relative_tolerance;
        if(P.reduce_mode == 0 || sizeof(R) == sizeof(double) || P.preconditioner != 0) {
            lastSolve = pcg_reference<R>(A, Avals, rhs, pressure, tolf, P.max_cg_iteration, P.preconditioner, nthreads());
            return;
        }
        std::vector<float> valsF(Avals.begin(), Avals.end());
        std::vector<float> rhsF(rhs.begin(), rhs.end());
        const int mode = P.pcg_mode & kPcgModeMask;
        const bool two = (P.pcg_mode & kPcgSingleReduction) == 0;
        if(mode == 0) {
            std::vector<float> x;
            lastSolve = pcg_canonical_any<float>(A, valsF, Adiag, rhsF, x, (float)tolf, P.max_cg_iteration, two);
            for(size_t i = 0; i < x.size(); ++i) pressure[i] = (R)x[i];
        } else if(mode == 1) {
            std::vector<double> x, r64(rhsF.begin(), rhsF.end());
            lastSolve = pcg_canonical_any<double>(A, valsF, Adiag, r64, x, (double)P.cg_relative_tolerance,
                                                  P.max_cg_iteration, two);
            for(size_t i = 0; i < x.size(); ++i) pressure[i] = (R)(float)x[i];
        } else {
            std::vector<double> x;
            lastSolve = pcg_refined(A, valsF, Adiag, rhsF, x, P.refine_inner_tolerance, (double)P.refine_tolerance,
                                    P.max_cg_iteration, two);
            for(size_t i = 0; i < x.size(); ++i) pressure[i] = (R)(float)x[i];
        }
    }

    // PIC_Solver::updateProjectedVelocity (PIC_Solver.cpp:911-981), weights = 1
    void updateVelocity(R dt) {
        for(int d = 0; d < 3; ++d) std::fill(valid[d].d.begin(), valid[d].d.end(), 0);
        for(int k = 0; k < G[2]; ++k)
            for(int j = 0; j < G[1]; ++j)
                for(int i = 0; i < G[0]; ++i) {
                    R pc = phi(i, j, k);
                    R pl = i > 0 ? phi(i - 1, j, k) : R(0);
                    R pb = j > 0 ? phi(i, j - 1, k) : R(0);
                    R pn = k > 0 ? phi(i, j, k - 1) : R(0);
                    R prc = pc < 0 ? pressure[activeIdx(i, j, k)] : R(0);
                    R prl = pl < 0 ? pressure[activeIdx(i - 1, j, k)] : R(0);
                    R prb = pb < 0 ? pressure[activeIdx(i, j - 1, k)] : R(0);
                    R prn = pn < 0 ? pressure[activeIdx(i, j, k - 1)] : R(0);
                    if(i > 0 && (pc < 0 || pl < 0) && faceWeight(0, i, j, k) > 0) {
                        R th = smax(R(0.01), fraction_inside(pl, pc));
                        u[0](i, j, k) -= dt * (prc - prl) / th; valid[0](i, j, k) = 1;
                    }
                    if(j > 0 && (pc < 0 || pb < 0) && faceWeight(1, i, j, k) > 0) {
                        R th = smax(R(0.01), fraction_inside(pb, pc));
                        u[1](i, j, k) -= dt * (prc - prb) / th; valid[1](i, j, k) = 1;
                    }
                    if(k > 0 && (pc < 0 || pn < 0) && faceWeight(2, i, j, k) > 0) {
                        R th = smax(R(0.01), fraction_inside(pn, pc));
                        u[2](i, j, k) -= dt * (prc - prn) / th; valid[2](i, j, k) = 1;
                    }
                }
        for(int d = 0; d < 3; ++d)
            for(size_t j = 0; j < u[d].size(); ++j) if(valid[d].d[j] == 0) u[d].d[j] = 0;
    }

    // ArrayHelpers::interpolateGradientValue 3D (ArrayHelpers.cpp:275-302)
    static void gradValue(const R pt[3], const Arr3<R>& a, R cellSize, R out[3]) {
        int i, j, k; R fi, fj, fk;
        get_barycentric(pt[0], i, fi, 0, a.sx);
        get_barycentric(pt[1], j, fj, 0, a.sy);
        get_barycentric(pt[2], k, fk, 0, a.sz);
        R v000 = a(i, j, k), v001 = a(i, j, k + 1), v010 = a(i, j + 1, k), v011 = a(i, j + 1, k + 1);
        R v100 = a(i + 1, j, k), v101 = a(i + 1, j, k + 1), v110 = a(i + 1, j + 1, k), v111 = a(i + 1, j + 1, k + 1);
        const R o = R(1.0);
        R w[8][3] = {
            {-(o - fj) * (o - fk), -(o - fi) * (o - fk), -(o - fi) * (o - fj)},
            {-(o - fj) * fk, -(o - fi) * fk, (o - fi) * (o - fj)},
            {-fj * (o - fk), (o - fi) * (o - fk), -(o - fi) * fj},
            {-fj * fk, (o - fi) * fk, (o - fi) * fj},
            {(o - fj) * (o - fk), -fi * (o - fk), -fi * (o - fj)},
            {(o - fj) * fk, -fi * fk, fi * (o - fj)},
            {fj * (o - fk), fi * (o - fk), -fi * fj},
            {fj * fk, fi * fk, fi * fj}};
        R v[8] = {v000, v001, v010, v011, v100, v101, v110, v111};
        for(int c = 0; c < 3; ++c) {
            R s = v[0] * w[0][c];
            for(int q = 1; q < 8; ++q) s = s + v[q] * w[q][c];
            out[c] = s / cellSize;
        }
    }

    // FLIP_Solver::mapGrid2Particles (FLIP_Solver.cpp:99-111) with
    // getVelocityChangesFromGrid (:125-133); APIC (APIC_Solver.cpp:95-117) and AFLIP
    // (AFLIP_Solver.cpp:94-132) variants; PIC takes the grid velocity (ratio 0).
    void mapG2P() {
        int kind = P.solver_kind;
        R ratio = (R)P.pic_flip_ratio;
#pragma omp parallel for schedule(static) if(nthreads() > 1)
        for(long long p = 0; p < (long long)pos.size(); ++p) {
            R g[3]; gridCoord(pos[p], g);
            R gv[3], dgv[3];
            for(int d = 0; d < 3; ++d) gv[d] = velFromGrid(g, d, u);
            if(kind == 1) { // APIC
                for(int d = 0; d < 3; ++d) vel[p][d] = gv[d];
            } else {
                for(int d = 0; d < 3; ++d) dgv[d] = velFromGrid(g, d, dV);
                for(int d = 0; d < 3; ++d) vel[p][d] = (R(1.0) - ratio) * gv[d] + ratio * (vel[p][d] + dgv[d]);
            }
            if(kind == 1 || kind == 2) {
                for(int d = 0; d < 3; ++d) {
                    R pt[3]; for(int a = 0; a < 3; ++a) pt[a] = g[a] - (a == d ? R(0) : R(0.5));
                    R gc[3]; gradValue(pt, u[d], dx, gc);
                    R* C = &Cmat[(size_t)p * 9 + d * 3];
                    if(kind == 1) { C[0] = gc[0]; C[1] = gc[1]; C[2] = gc[2]; }
                    else {
                        R dc[3]; gradValue(pt, dV[d], dx, dc);
                        for(int c = 0; c < 3; ++c) C[c] = (R(1.0) - ratio) * gc[c] + ratio * (C[c] + dc[c]);
                    }
                }
            }
        }
    }

    std::vector<Arr3<R>> snap; // optional stage snapshots for stage-level diffs

    static double now() {
#ifdef _OPENMP
        return omp_get_wtime();
#else
        return 0.0;
#endif
    }

    // One iteration of PIC_Solver::advanceFrame's sub-step loop (PIC_Solver.cpp:277-305)
    // followed by FLIP_Solver::advanceVelocity (FLIP_Solver.cpp:42-53).
    void step(orc_step_stats* st) {
        if(frameTime >= frameDuration) frameTime = R(0);
        double t0 = now();
        R substep = timestepCFL();
        R remaining = frameDuration - frameTime;
        if(frameTime + substep >= frameDuration) substep = remaining;
        else if(frameTime + R(1.5) * substep >= frameDuration) substep = remaining * R(0.5);
        moveParticles(substep);
        double t1 = now();
        if(P.correct_position) {
            // PIC_Solver::advanceFrame: moveParticles, correctParticlePositions (PIC_Solver.cpp:292-293)
            sortParticlesByCell();
            correctPositions(substep);
        }
        if(P.sort_each_step || P.correct_position) sortParticlesByCell();
        double t2 = now();
        int kind = P.solver_kind;
        // PIC_Solver::advanceVelocity (PIC_Solver.cpp:332-338): advect the grid velocity,
        // gravity, projection, extrapolation; the particles only carry the fluid SDF
        if(kind == 3) advectGrid(substep);
        else splatParticles();
        double t3 = now();
        if(kind != 1 && kind != 3) {
            extrapolateAll(); // APIC goes straight to gravity (APIC_Solver.cpp:42-49)
            if(gridBoundary) constrainGridVelocity();  // FLIP_Solver.cpp:46
        }
        if(kind == 0 || kind == 2) for(int d = 0; d < 3; ++d) old[d].d = u[d].d;   // backupGridVelocity
        double t4 = now();
        addGravity(substep);
        computeFluidSDF();
        double t5 = now();
        computeSystem(substep);
        double t6 = now();
        solveSystem();
        double t7 = now();
        updateVelocity(substep);
        extrapolateAll();
        if(gridBoundary) constrainGridVelocity();
        double t8 = now();
        if(kind == 0 || kind == 2)
            for(int d = 0; d < 3; ++d)
                for(size_t i = 0; i < u[d].size(); ++i) dV[d].d[i] = u[d].d[i] - old[d].d[i];
        if(kind != 3) mapG2P();
        double t9 = now();
        frameTime += substep;
        ++substepIndex;
        if(st) {
            st->dt = (double)substep; st->frame_time = (double)frameTime;
            st->frame_finished = frameTime >= frameDuration ? 1 : 0;
            st->pcg_iterations = lastSolve.iterations; st->pcg_residual = lastSolve.residual;
            st->pcg_success = lastSolve.success ? 1 : 0; st->n_active = nActive; st->outer_iterations = lastSolve.outer;
            st->zero_phi_cells = zeroPhiCells;
            st->t_move = t1 - t0; st->t_sort = t2 - t1; st->t_p2g = t3 - t2; st->t_extrap = (t4 - t3) + (t8 - t7) * 0.5;
            st->t_sdf = t5 - t4; st->t_system = t6 - t5; st->t_solve = t7 - t6; st->t_update = (t8 - t7) * 0.5; st->t_g2p = t9 - t8;
        }
    }
};

// ----------------------------------------------------------------------------------
// Uniform-grid cell sort, NeighborSearch and Morton z-sort (config 3)
// ----------------------------------------------------------------------------------

// Morton3D 64-bit encode as m3D_e_sLUT<uint_fast64_t, uint_fast32_t> computes it
// (Morton/Morton3D.h:54-66, Morton.h:51): bytes of x/y/z are bit-interleaved 8 at a time
// (x -> bit 3b, y -> 3b+1, z -> 3b+2) and each byte group is shifted in by 24 bits, so
// only the three lowest bytes of each coordinate survive in the 64-bit result.
static inline uint64_t spread8(uint64_t b) {
    uint64_t r = 0;
    for(int i = 0; i < 8; ++i) if(b & (1ull << i)) r |= 1ull << (3 * i);
    return r;
}
static uint64_t morton3d(uint64_t x, uint64_t y, uint64_t z) {
    uint64_t ans = 0;
    for(int i = (int)sizeof(uint_fast32_t); i > 0; --i) {
        unsigned shift = (unsigned)(i - 1) * 8;
        ans = (ans << 24) | ((spread8((z >> shift) & 0xFF) << 2) | (spread8((y >> shift) & 0xFF) << 1) | spread8((x >> shift) & 0xFF));
    }
    return ans;
}

// NeighborSearch::cell_index (NeighborSearch.cpp:44-52), SHIFT_POSITION = 1.2345
// (DataStructures.h:32); inv_cell_size = float(1.0 / r) (NeighborSearch.cpp:32-34).
static inline void ns_key(const float* x, float inv, int k[3]) {
    for(int d = 0; d < 3; ++d) {
        float t = x[d] - (float)1.2345;
        k[d] = t >= 0 ? (int)(inv * t) : (int)(inv * t) - 1;
    }
}

} // namespace orc

using namespace orc;

// ----------------------------------------------------------------------------------
// C API (ctypes)
// ----------------------------------------------------------------------------------
struct orc_handle {
    bool dbl = false;
    std::unique_ptr<FlipOracle<float>> f;
    std::unique_ptr<FlipOracle<double>> d;
};

extern "C" {

int orc_set_threads(int n) {
#ifdef _OPENMP
    if(n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

void* orc_create(const orc_params* p, int use_double) {
    auto* h = new orc_handle();
    h->dbl = use_double != 0;
    if(h->dbl) h->d = std::make_unique<FlipOracle<double>>(*p);
    else h->f = std::make_unique<FlipOracle<float>>(*p);
    return h;
}

void orc_destroy(void* hp) { delete (orc_handle*)hp; }

void orc_grid_dims(void* hp, int32_t* g) {
    auto* h = (orc_handle*)hp;
    for(int d = 0; d < 3; ++d) g[d] = h->dbl ? h->d->G[d] : h->f->G[d];
}

} // extern "C"
template<class R> static void set_parts(FlipOracle<R>& o, const float* pos, const float* vel, uint32_t n) {
    o.pos.resize(n); o.vel.resize(n); o.pid.resize(n);
    bool aff = o.P.solver_kind == 1 || o.P.solver_kind == 2;
    o.Cmat.assign(aff ? (size_t)n * 9 : 0, R(0));
    for(uint32_t i = 0; i < n; ++i) {
        o.pos[i] = V3<R>{(R)pos[3 * i], (R)pos[3 * i + 1], (R)pos[3 * i + 2]};
        o.vel[i] = V3<R>{(R)vel[3 * i], (R)vel[3 * i + 1], (R)vel[3 * i + 2]};
        o.pid[i] = i;
    }
}
extern "C" {
void orc_set_particles(void* hp, const float* pos, const float* vel, uint32_t n) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) set_parts(*h->d, pos, vel, n); else set_parts(*h->f, pos, vel, n);
}

// Particles in original (input) order; positions / velocities as float (or double)
} // extern "C"
template<class R, class T> static void get_parts(FlipOracle<R>& o, T* pos, T* vel) {
    for(size_t i = 0; i < o.pos.size(); ++i) {
        uint32_t id = o.pid[i];
        pos[3 * id] = (T)o.pos[i].x; pos[3 * id + 1] = (T)o.pos[i].y; pos[3 * id + 2] = (T)o.pos[i].z;
        vel[3 * id] = (T)o.vel[i].x; vel[3 * id + 1] = (T)o.vel[i].y; vel[3 * id + 2] = (T)o.vel[i].z;
    }
}
extern "C" {
void orc_get_particles(void* hp, float* pos, float* vel) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) get_parts(*h->d, pos, vel); else get_parts(*h->f, pos, vel);
}
void orc_get_particles_f64(void* hp, double* pos, double* vel) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) get_parts(*h->d, pos, vel); else get_parts(*h->f, pos, vel);
}
// Particle order currently held (ids), for sort parity
void orc_get_particle_ids(void* hp, uint32_t* ids) {
    auto* h = (orc_handle*)hp;
    auto& v = h->dbl ? h->d->pid : h->f->pid;
    std::memcpy(ids, v.data(), v.size() * sizeof(uint32_t));
}

// which: 0..2 face velocity u/v/w, 3 fluid SDF, 4 pressure on cells (0 where not
// active), 5..7 old (backup) face velocity, 8 active index + 1 on cells (0 = inactive)
} // extern "C"
template<class R, class T> static int get_grid(FlipOracle<R>& o, int which, T* out) {
    if(which >= 0 && which < 3) { for(size_t i = 0; i < o.u[which].size(); ++i) out[i] = (T)o.u[which].d[i]; return 0; }
    if(which >= 5 && which < 8) { for(size_t i = 0; i < o.old[which - 5].size(); ++i) out[i] = (T)o.old[which - 5].d[i]; return 0; }
    if(which == 3) { for(size_t i = 0; i < o.phi.size(); ++i) out[i] = (T)o.phi.d[i]; return 0; }
    if(which == 4) {
        for(size_t i = 0; i < o.phi.size(); ++i) out[i] = o.phi.d[i] < 0 ? (T)o.pressure[o.activeIdx.d[i]] : (T)0;
        return 0;
    }
    if(which == 8) {
        for(size_t i = 0; i < o.phi.size(); ++i) out[i] = o.phi.d[i] < 0 ? (T)(o.activeIdx.d[i] + 1) : (T)0;
        return 0;
    }
    if(which >= 9 && which < 12) {
        const int d = which - 9;
        for(size_t i = 0; i < o.u[d].size(); ++i) out[i] = o.gridBoundary ? (T)o.weight[d].d[i] : (T)1;
        return 0;
    }
    if(which == 12) {
        const size_t nn = (size_t)(o.G[0] + 1) * (o.G[1] + 1) * (o.G[2] + 1);
        for(size_t i = 0; i < nn; ++i) out[i] = o.gridBoundary ? (T)o.nodeSdf.d[i] : (T)0;
        return 0;
    }
    return -1;
}
extern "C" {
int orc_get_grid(void* hp, int which, float* out) {
    auto* h = (orc_handle*)hp;
    return h->dbl ? get_grid(*h->d, which, out) : get_grid(*h->f, which, out);
}
int orc_get_grid_f64(void* hp, int which, double* out) {
    auto* h = (orc_handle*)hp;
    return h->dbl ? get_grid(*h->d, which, out) : get_grid(*h->f, which, out);
}
// Set face velocities (for stage tests that start from a given grid)
int orc_set_grid(void* hp, int which, const float* in) {
    auto* h = (orc_handle*)hp;
    if(which < 0 || which > 2) return -1;
    if(h->dbl) { auto& a = h->d->u[which]; for(size_t i = 0; i < a.size(); ++i) a.d[i] = in[i]; }
    else { auto& a = h->f->u[which]; for(size_t i = 0; i < a.size(); ++i) a.d[i] = in[i]; }
    return 0;
}

// Boundary objects besides the domain box (bnn_flip_set_boundaries semantics)
int orc_set_boundaries(void* hp, const orc_boundary_object* objs, uint32_t n, int updateGrid) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) h->d->setBoundaries(objs, n, updateGrid != 0); else h->f->setBoundaries(objs, n, updateGrid != 0);
    return 0;
}

int orc_step(void* hp, orc_step_stats* st) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) h->d->step(st); else h->f->step(st);
    return 0;
}

// The cell sort and P2G alone (FLIP_Solver::mapParticles2Grid on the current particles),
// for analytic checks of the transfer
int orc_p2g_only(void* hp) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) { h->d->sortParticlesByCell(); h->d->splatParticles(); }
    else { h->f->sortParticlesByCell(); h->f->splatParticles(); }
    return 0;
}

// Pressure system of the last step as CSR (rows = active cells) plus rhs
uint32_t orc_system_nnz(void* hp) {
    auto* h = (orc_handle*)hp;
    return h->dbl ? (uint32_t)h->d->A.colIndex.size() : (uint32_t)h->f->A.colIndex.size();
}
void orc_get_system(void* hp, uint32_t* rowStart, uint32_t* colIndex, float* vals, float* rhs) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) return;
    auto& o = *h->f;
    std::memcpy(rowStart, o.A.rowStart.data(), o.A.rowStart.size() * 4);
    std::memcpy(colIndex, o.A.colIndex.data(), o.A.colIndex.size() * 4);
    for(size_t i = 0; i < o.Avals.size(); ++i) vals[i] = o.Avals[i];
    for(size_t i = 0; i < o.rhs.size(); ++i) rhs[i] = o.rhs[i];
}

// Standalone PCG on a CSR system (rows column-sorted), in the chosen arithmetic.
// mode: 0 canonical FP32, 1 canonical FP64, 2 refined, 3 reference FP32 (precond 0/1/2),
// 4 reference FP64; modes 0-2 take PCGSolver's two-reduction step order unless
// kPcgSingleReduction is OR-ed in.
int orc_pcg(uint32_t n, const uint32_t* rowStart, const uint32_t* colIndex, const float* vals, const float* rhs,
            float tol, uint32_t maxIter, int mode, int precond, float innerTol, double* x_out, uint32_t* iters,
            double* resid, uint32_t* outer) {
    CSR A;
    A.n = n;
    A.rowStart.assign(rowStart, rowStart + n + 1);
    A.colIndex.assign(colIndex, colIndex + rowStart[n]);
    std::vector<float> v(vals, vals + rowStart[n]);
    std::vector<float> diag(n, 0.0f);
    for(uint32_t r = 0; r < n; ++r)
        for(uint32_t j = rowStart[r]; j < rowStart[r + 1]; ++j) if(colIndex[j] == r) diag[r] = vals[j];
    std::vector<float> b(rhs, rhs + n);
    PCGResult res;
    const bool two = (mode & kPcgSingleReduction) == 0;
    mode &= kPcgModeMask;
    if(mode == 0) {
        std::vector<float> x; res = pcg_canonical_any<float>(A, v, diag, b, x, tol, maxIter, two);
        for(uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
    } else if(mode == 1) {
        std::vector<double> x, b64(b.begin(), b.end());
        res = pcg_canonical_any<double>(A, v, diag, b64, x, (double)tol, maxIter, two);
        for(uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
    } else if(mode == 2) {
        std::vector<double> x; res = pcg_refined(A, v, diag, b, x, innerTol, (double)tol, maxIter, two);
        for(uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
    } else if(mode == 3) {
        std::vector<float> x; res = pcg_reference<float>(A, v, b, x, tol, maxIter, precond, 1);
        for(uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
    } else {
        std::vector<double> v64(v.begin(), v.end()), b64(b.begin(), b.end()), x;
        res = pcg_reference<double>(A, v64, b64, x, (double)tol, maxIter, precond, 1);
        for(uint32_t i = 0; i < n; ++i) x_out[i] = x[i];
    }
    *iters = res.iterations; *resid = res.residual; *outer = res.outer;
    return res.success ? 0 : 1;
}

// Canonical dot product (exposed so tests can pin the reduction order)
double orc_dot_canonical_f32(const float* a, const float* b, uint64_t n) { return dot_canonical(a, b, (size_t)n); }

// Grid cell index (Grid::getCellIdx, Grid.h:156-162; truncation toward zero) and the
// canonical sorted index: particles by linear cell id, ties in input order (what
// Grid::getParticleIdxSortedByCell returns when collectIndexToCells runs on one thread).
// Cells outside the grid are clamped onto its border; out_of_range counts them.
uint32_t orc_cell_sort(const float* pos, uint32_t n, const float* bmin, float cellSize, const int32_t* ncells,
                       uint32_t* cellId, uint32_t* sortedIdx, uint32_t* cellStart) {
    uint32_t oor = 0;
    size_t C = (size_t)ncells[0] * ncells[1] * ncells[2];
    std::vector<uint32_t> start(C + 1, 0);
    for(uint32_t p = 0; p < n; ++p) {
        int c[3];
        for(int d = 0; d < 3; ++d) {
            c[d] = (int)((pos[3 * p + d] - bmin[d]) / cellSize);
            if(c[d] < 0 || c[d] >= ncells[d]) { ++oor; c[d] = c[d] < 0 ? 0 : ncells[d] - 1; }
        }
        cellId[p] = (uint32_t)(((size_t)c[2] * ncells[1] + c[1]) * ncells[0] + c[0]);
        start[cellId[p] + 1]++;
    }
    for(size_t c = 0; c < C; ++c) start[c + 1] += start[c];
    if(cellStart) std::memcpy(cellStart, start.data(), (C + 1) * 4);
    for(uint32_t p = 0; p < n; ++p) sortedIdx[start[cellId[p]]++] = p;
    return oor;
}

// NeighborSearch::z_value (NeighborSearch.cpp:57-67) of each point's cell_index, and the
// z_sort permutation (NeighborSearch.cpp:72-86) made canonical: ties in input order.
void orc_z_sort(const float* pos, uint32_t n, float radius, uint64_t* zval, uint32_t* perm) {
    float inv = (float)(1.0 / (double)radius);
    for(uint32_t p = 0; p < n; ++p) {
        int k[3]; ns_key(pos + 3 * p, inv, k);
        uint64_t c[3];
        for(int d = 0; d < 3; ++d) c[d] = (uint64_t)((int64_t)k[d] - ((int64_t)std::numeric_limits<int>::lowest() + 1));
        zval[p] = morton3d(c[0], c[1], c[2]);
    }
    std::iota(perm, perm + n, 0u);
    std::stable_sort(perm, perm + n, [&](uint32_t a, uint32_t b) { return zval[a] < zval[b]; });
}

// NeighborSearch::find_neighbors + query3D (NeighborSearch.cpp:219-226,530-692), one
// point set searching itself: for every point all others with |x-y|^2 < r^2 (strict,
// squared distance summed as (dx*dx + dy*dy) + dz*dz), over the 27 hash cells.  Each list
// is returned sorted ascending (the reference's order depends on its thread schedule).
// Pass offsets == nullptr to only count.  Returns the total number of entries.
uint64_t orc_neighbors(const float* pos, uint32_t n, float radius, uint64_t* offsets, uint32_t* idx) {
    float inv = (float)(1.0 / (double)radius);
    float r2 = radius * radius;
    struct KH { size_t operator()(const uint64_t k) const { return std::hash<uint64_t>()(k * 0x9E3779B97F4A7C15ull); } };
    auto pack = [](int a, int b, int c) {
        return ((uint64_t)(uint32_t)(a + (1 << 20)) << 42) | ((uint64_t)(uint32_t)(b + (1 << 20)) << 21) | (uint64_t)(uint32_t)(c + (1 << 20));
    };
    std::vector<int> keys(3 * (size_t)n);
    std::unordered_map<uint64_t, std::vector<uint32_t>, KH> cells;
    for(uint32_t p = 0; p < n; ++p) {
        ns_key(pos + 3 * p, inv, &keys[3 * (size_t)p]);
        cells[pack(keys[3 * p], keys[3 * p + 1], keys[3 * p + 2])].push_back(p);
    }
    std::vector<uint64_t> counts(n, 0);
    // pass 0 counts, pass 1 writes each (sorted) list at its offset
    for(int pass = 0; pass < (offsets ? 2 : 1); ++pass) {
#pragma omp parallel
        {
            std::vector<uint32_t> loc;
#pragma omp for schedule(dynamic, 1024)
            for(long long pl = 0; pl < (long long)n; ++pl) {
                uint32_t p = (uint32_t)pl;
                const float* xa = pos + 3 * (size_t)p;
                loc.clear();
                for(int a = -1; a <= 1; ++a)
                    for(int b = -1; b <= 1; ++b)
                        for(int c = -1; c <= 1; ++c) {
                            auto it = cells.find(pack(keys[3 * p] + a, keys[3 * p + 1] + b, keys[3 * p + 2] + c));
                            if(it == cells.end()) continue;
                            for(uint32_t q : it->second) {
                                if(q == p) continue;
                                const float* xb = pos + 3 * (size_t)q;
                                float t0 = xa[0] - xb[0], t1 = xa[1] - xb[1], t2 = xa[2] - xb[2];
                                float l2 = t0 * t0 + t1 * t1 + t2 * t2;
                                if(l2 < r2) loc.push_back(q);
                            }
                        }
                if(pass == 0) counts[p] = loc.size();
                else {
                    std::sort(loc.begin(), loc.end());
                    std::memcpy(idx + offsets[p], loc.data(), loc.size() * 4);
                }
            }
        }
        if(pass == 0 && offsets) {
            uint64_t o = 0;
            for(uint32_t p = 0; p < n; ++p) { offsets[p] = o; o += counts[p]; }
            offsets[n] = o;
        }
    }
    uint64_t total = 0;
    for(uint32_t p = 0; p < n; ++p) total += counts[p];
    return total;
}

// Grid::getNeighborList(positions, list, d2, span) (Grid.cpp:229-279) for one query point:
// every point in the 27 cells around it with 0 < |x-y|^2 < d2 (used by the Grid test).
uint32_t orc_grid_neighbor_list(const float* pos, uint32_t n, const float* bmin, float cellSize, const int32_t* ncells,
                                const float* q, float d2, int with_distance, uint32_t* out) {
    uint32_t cnt = 0;
    int c[3];
    for(int d = 0; d < 3; ++d) c[d] = (int)((q[d] - bmin[d]) / cellSize);
    for(int lk = -1; lk <= 1; ++lk)
        for(int lj = -1; lj <= 1; ++lj)
            for(int li = -1; li <= 1; ++li) {
                int cc[3] = {c[0] + li, c[1] + lj, c[2] + lk};
                bool ok = true;
                for(int d = 0; d < 3; ++d) if(cc[d] < 0 || cc[d] >= ncells[d]) ok = false;
                if(!ok) continue;
                for(uint32_t p = 0; p < n; ++p) {
                    int pc[3];
                    for(int d = 0; d < 3; ++d) pc[d] = (int)((pos[3 * p + d] - bmin[d]) / cellSize);
                    if(pc[0] != cc[0] || pc[1] != cc[1] || pc[2] != cc[2]) continue;
                    if(with_distance) {
                        float t0 = q[0] - pos[3 * p], t1 = q[1] - pos[3 * p + 1], t2 = q[2] - pos[3 * p + 2];
                        float l2 = (t0 * t0 + t1 * t1) + t2 * t2;
                        if(!(l2 > 0 && l2 < d2)) continue;
                    }
                    out[cnt++] = p;
                }
            }
    return cnt;
}

// Grid::setCellSize cell counts (Grid.cpp:38-55): ceil((bMax - bMin) / cellSize) in float
void orc_grid_ncells(const float* bmin, const float* bmax, float cellSize, int32_t* out) {
    for(int d = 0; d < 3; ++d) out[d] = (int32_t)(uint32_t)std::ceil((bmax[d] - bmin[d]) / cellSize);
}

} // extern "C"

extern "C" {
// ArrayHelpers::interpolateValueLinear of face component d at grid coordinates g (for the
// analytic interpolation checks)
double orc_interp_face(void* hp, int d, double gx, double gy, double gz) {
    auto* h = (orc_handle*)hp;
    if(h->dbl) { double g[3] = {gx, gy, gz}; return h->d->velFromGrid(g, d, h->d->u); }
    float g[3] = {(float)gx, (float)gy, (float)gz};
    return (double)h->f->velFromGrid(g, d, h->f->u);
}
} // extern "C"

// Single-rank PETSc/MPI/METIS stand-in for building the reference (PIGFEM
// 4.6.1) as a CPU oracle.  Test infrastructure only: nothing in the product
// links this file.  See include/petsc_shim.h for what each object models.
#include "petsc_shim.h"
#include "metis.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <string>
#include <vector>

namespace {

[[noreturn]] void shim_fail(const char* what) {
    fprintf(stderr, "[pg-ref-shim] unsupported call on a single rank: %s\n", what);
    abort();
}

double now_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

double g_ksp_seconds = 0.0;
long g_ksp_solves = 0;
long g_snes_iterations = 0;
int g_snes_verbose = 0;

}  // namespace

// --------------------------------------------------------------------------
// MPI (one rank)
// --------------------------------------------------------------------------
extern "C" {
int MPI_Init(int*, char***) { return 0; }
int MPI_Initialized(int* flag) { *flag = 1; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
int MPI_Barrier(MPI_Comm) { return 0; }
int MPI_Abort(MPI_Comm, int code) { fprintf(stderr, "MPI_Abort(%d)\n", code); abort(); }
static int copy_buf(const void* s, void* r, int count, MPI_Datatype dt) {
    if (s != MPI_IN_PLACE && s != r && count > 0) memmove(r, s, (size_t)count * (size_t)dt);
    return 0;
}
int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Reduce(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, int, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Scan(const void* s, void* r, int c, MPI_Datatype dt, MPI_Op, MPI_Comm) { return copy_buf(s, r, c, dt); }
int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
int MPI_Gather(const void* s, int sc, MPI_Datatype sdt, void* r, int, MPI_Datatype, int, MPI_Comm) { return copy_buf(s, r, sc, sdt); }
int MPI_Allgather(const void* s, int sc, MPI_Datatype sdt, void* r, int, MPI_Datatype, MPI_Comm) { return copy_buf(s, r, sc, sdt); }
int MPI_Gatherv(const void* s, int sc, MPI_Datatype sdt, void* r, const int*, const int* displs, MPI_Datatype rdt, int, MPI_Comm) {
    return copy_buf(s, (char*)r + (size_t)displs[0] * (size_t)rdt, sc, sdt);
}
int MPI_Allgatherv(const void* s, int sc, MPI_Datatype sdt, void* r, const int*, const int* displs, MPI_Datatype rdt, MPI_Comm) {
    return copy_buf(s, (char*)r + (size_t)displs[0] * (size_t)rdt, sc, sdt);
}
int MPI_Alltoall(const void* s, int sc, MPI_Datatype sdt, void* r, int, MPI_Datatype, MPI_Comm) { return copy_buf(s, r, sc, sdt); }
int MPI_Isend(const void*, int count, MPI_Datatype, int, int, MPI_Comm, MPI_Request* req) {
    if (count > 0) shim_fail("MPI_Isend");
    *req = 0; return 0;
}
int MPI_Send(const void*, int count, MPI_Datatype, int, int, MPI_Comm) { if (count > 0) shim_fail("MPI_Send"); return 0; }
int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { shim_fail("MPI_Recv"); }
int MPI_Probe(int, int, MPI_Comm, MPI_Status*) { shim_fail("MPI_Probe"); }
int MPI_Get_count(const MPI_Status* st, MPI_Datatype dt, int* count) { *count = st ? st->count_bytes / dt : 0; return 0; }
int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
int MPI_Type_create_struct(int count, const int* bl, const MPI_Aint*, const MPI_Datatype* types, MPI_Datatype* nt) {
    int bytes = 0;
    for (int i = 0; i < count; ++i) bytes += bl[i] * types[i];
    *nt = bytes;
    return 0;
}
int MPI_Type_commit(MPI_Datatype*) { return 0; }
int MPI_Type_free(MPI_Datatype*) { return 0; }
double MPI_Wtime(void) { return now_s(); }

int METIS_SetDefaultOptions(idx_t*) { return METIS_OK; }
int METIS_PartMeshDual(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, real_t*, idx_t*, idx_t*, idx_t*, idx_t*) {
    shim_fail("METIS_PartMeshDual");
}
int METIS_PartMeshNodal(idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, real_t*, idx_t*, idx_t*, idx_t*, idx_t*) {
    shim_fail("METIS_PartMeshNodal");
}
}  // extern "C"

// --------------------------------------------------------------------------
// Objects
// --------------------------------------------------------------------------
struct _p_Vec {
    std::vector<double> a;
};
struct _p_IS {
    std::vector<PetscInt> idx;
};
struct _p_VecScatter {
    bool to_all = false;
    std::vector<PetscInt> from, to;
};

// Envelope (skyline) LDL^T factor of a symmetric matrix in a reverse
// Cuthill-McKee ordering.  No pivoting: the matrices it sees are symmetric
// stiffness matrices (SPD, or mildly indefinite under cohesive softening).
struct SkylineLDLT {
    int n = 0;
    std::vector<int> perm, iperm;      // perm[new] = old
    std::vector<int> first;            // first column of row i (permuted)
    std::vector<size_t> start;         // offset of row i's envelope
    std::vector<double> env;           // L entries (row i: columns first[i]..i-1)
    std::vector<double> d;
    bool ok = false;

    void factor(const struct _p_Mat* A);
    void solve(const double* b, double* x) const;
};

struct _p_Mat {
    int m = 0, n = 0;
    bool dense = false;
    std::vector<std::vector<PetscInt>> cols;
    std::vector<std::vector<double>> vals;
    std::vector<double> dd;  // dense storage, column major
    long version = 0;
    // Factor matrices (MatGetFactor) point at their source.
    Mat factor_of = nullptr;
    SkylineLDLT* fac = nullptr;

    void ensure_sparse(int mm, int nn) {
        m = mm; n = nn;
        cols.assign(m, {});
        vals.assign(m, {});
    }
};

struct _p_PC {
    std::string type;
};
struct _p_KSP {
    Mat A = nullptr;
    _p_PC pc;
    std::string type;
    SkylineLDLT fac;
    long fac_version = -1;
    Mat fac_mat = nullptr;
};
struct _p_SNES {
    _p_KSP ksp;
    Vec r = nullptr;
    Mat J = nullptr;
    SNESFunctionFn f = nullptr;
    void* fctx = nullptr;
    SNESJacobianFn jac = nullptr;
    void* jctx = nullptr;
    SNESMonitorFn mon = nullptr;
    void* mctx = nullptr;
    double atol = 1e-50, rtol = 1e-8, stol = 1e-8;
    int maxit = 50;
    int maxf = 10000;
    double fnorm = 0.0;
    int its = 0;
    SNESConvergedReason reason = SNES_CONVERGED_ITERATING;
};

// ---- skyline LDL^T --------------------------------------------------------
static void rcm_order(const _p_Mat* A, std::vector<int>& perm) {
    const int n = A->m;
    std::vector<int> deg(n);
    for (int i = 0; i < n; ++i) deg[i] = (int)A->cols[i].size();
    std::vector<char> seen(n, 0);
    std::vector<int> order;
    order.reserve(n);
    while ((int)order.size() < n) {
        // pseudo-peripheral start: unseen node of minimum degree
        int s = -1;
        for (int i = 0; i < n; ++i)
            if (!seen[i] && (s < 0 || deg[i] < deg[s])) s = i;
        std::deque<int> q;
        q.push_back(s);
        seen[s] = 1;
        while (!q.empty()) {
            int v = q.front();
            q.pop_front();
            order.push_back(v);
            std::vector<int> nb;
            for (PetscInt c : A->cols[v])
                if (c != v && !seen[c]) { seen[c] = 1; nb.push_back(c); }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
            for (int c : nb) q.push_back(c);
        }
    }
    std::reverse(order.begin(), order.end());
    perm = order;
}

void SkylineLDLT::factor(const _p_Mat* A) {
    n = A->m;
    rcm_order(A, perm);
    iperm.assign(n, 0);
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    first.assign(n, 0);
    for (int i = 0; i < n; ++i) {
        int f = i;
        for (PetscInt c : A->cols[perm[i]]) f = std::min(f, iperm[c]);
        first[i] = f;
    }
    // symmetric envelope: use row envelopes of the lower triangle
    start.assign(n + 1, 0);
    for (int i = 0; i < n; ++i) start[i + 1] = start[i] + (size_t)(i - first[i]);
    env.assign(start[n], 0.0);
    d.assign(n, 0.0);
    for (int i = 0; i < n; ++i) {
        const int oi = perm[i];
        const auto& cs = A->cols[oi];
        const auto& vs = A->vals[oi];
        for (size_t k = 0; k < cs.size(); ++k) {
            int j = iperm[cs[k]];
            if (j < i) env[start[i] + (j - first[i])] = vs[k];
            else if (j == i) d[i] = vs[k];
        }
    }
    // Crout: row i, columns j in [first[i], i)
    for (int i = 0; i < n; ++i) {
        double* Li = &env[start[i]];
        const int fi = first[i];
        for (int j = fi; j < i; ++j) {
            const int fj = first[j];
            const double* Lj = &env[start[j]];
            const int k0 = std::max(fi, fj);
            // Li[k] (k < j) holds t_ik = l_ik * d_k; Lj holds the final l_jk.
            double s = Li[j - fi];
            for (int k = k0; k < j; ++k) s -= Li[k - fi] * Lj[k - fj];
            Li[j - fi] = s;  // t_ij = l_ij * d_j
        }
        double di = d[i];
        for (int j = fi; j < i; ++j) {
            const double t = Li[j - fi];
            const double l = t / d[j];
            di -= t * l;
            Li[j - fi] = l;
        }
        d[i] = di;
    }
    ok = true;
}

void SkylineLDLT::solve(const double* b, double* x) const {
    std::vector<double> y(n);
    for (int i = 0; i < n; ++i) y[i] = b[perm[i]];
    for (int i = 0; i < n; ++i) {
        const double* Li = &env[start[i]];
        double s = y[i];
        for (int j = first[i]; j < i; ++j) s -= Li[j - first[i]] * y[j];
        y[i] = s;
    }
    for (int i = 0; i < n; ++i) y[i] /= d[i];
    for (int i = n - 1; i >= 0; --i) {
        const double* Li = &env[start[i]];
        const double yi = y[i];
        for (int j = first[i]; j < i; ++j) y[j] -= Li[j - first[i]] * yi;
    }
    for (int i = 0; i < n; ++i) x[perm[i]] = y[i];
}

// --------------------------------------------------------------------------
// PETSc API
// --------------------------------------------------------------------------
extern "C" {

PetscErrorCode PetscInitialize(int*, char***, const char*, const char*) { return 0; }
PetscErrorCode PetscFinalize(void) { return 0; }
PetscErrorCode MatFactorInfoInitialize(MatFactorInfo* info) { memset(info, 0, sizeof(*info)); return 0; }

// ---- Vec --------------------------------------------------------------
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt n, Vec* v) {
    *v = new _p_Vec;
    (*v)->a.assign(n > 0 ? n : 0, 0.0);
    return 0;
}
PetscErrorCode VecCreateMPI(MPI_Comm c, PetscInt n, PetscInt N, Vec* v) {
    return VecCreateSeq(c, n >= 0 ? n : N, v);
}
PetscErrorCode VecDestroy(Vec* v) { if (v && *v) { delete *v; *v = nullptr; } return 0; }
PetscErrorCode VecDuplicate(Vec v, Vec* out) { *out = new _p_Vec; (*out)->a.assign(v->a.size(), 0.0); return 0; }
PetscErrorCode VecZeroEntries(Vec v) { std::fill(v->a.begin(), v->a.end(), 0.0); return 0; }
PetscErrorCode VecSet(Vec v, PetscScalar a) { std::fill(v->a.begin(), v->a.end(), a); return 0; }
PetscErrorCode VecCopy(Vec x, Vec y) { y->a = x->a; return 0; }
PetscErrorCode VecAXPY(Vec y, PetscScalar a, Vec x) {
    for (size_t i = 0; i < y->a.size(); ++i) y->a[i] += a * x->a[i];
    return 0;
}
PetscErrorCode VecAYPX(Vec y, PetscScalar a, Vec x) {
    for (size_t i = 0; i < y->a.size(); ++i) y->a[i] = x->a[i] + a * y->a[i];
    return 0;
}
PetscErrorCode VecWAXPY(Vec w, PetscScalar a, Vec x, Vec y) {
    w->a.resize(x->a.size());
    for (size_t i = 0; i < x->a.size(); ++i) w->a[i] = a * x->a[i] + y->a[i];
    return 0;
}
PetscErrorCode VecScale(Vec v, PetscScalar a) { for (double& e : v->a) e *= a; return 0; }
PetscErrorCode VecDot(Vec x, Vec y, PetscScalar* val) {
    double s = 0.0;
    for (size_t i = 0; i < x->a.size(); ++i) s += x->a[i] * y->a[i];
    *val = s;
    return 0;
}
PetscErrorCode VecNorm(Vec x, NormType t, PetscReal* val) {
    double s = 0.0;
    if (t == NORM_1) { for (double e : x->a) s += std::fabs(e); }
    else if (t == NORM_INFINITY) { for (double e : x->a) s = std::max(s, std::fabs(e)); }
    else { for (double e : x->a) s += e * e; s = std::sqrt(s); }
    *val = s;
    return 0;
}
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar a, InsertMode mode) {
    if (i < 0) return 0;
    if ((size_t)i >= v->a.size()) shim_fail("VecSetValue out of range");
    if (mode == ADD_VALUES) v->a[i] += a; else v->a[i] = a;
    return 0;
}
PetscErrorCode VecSetValues(Vec v, PetscInt n, const PetscInt ix[], const PetscScalar y[], InsertMode mode) {
    for (PetscInt k = 0; k < n; ++k) VecSetValue(v, ix[k], y[k], mode);
    return 0;
}
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt ix[], PetscScalar y[]) {
    for (PetscInt k = 0; k < n; ++k) y[k] = v->a[ix[k]];
    return 0;
}
PetscErrorCode VecAssemblyBegin(Vec) { return 0; }
PetscErrorCode VecAssemblyEnd(Vec) { return 0; }
PetscErrorCode VecGetArray(Vec v, PetscScalar** a) { *a = v->a.data(); return 0; }
PetscErrorCode VecRestoreArray(Vec, PetscScalar** a) { *a = nullptr; return 0; }
PetscErrorCode VecGetArrayRead(Vec v, const PetscScalar** a) { *a = v->a.data(); return 0; }
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar** a) { *a = nullptr; return 0; }
PetscErrorCode VecGetSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n) { *n = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecGetOwnershipRange(Vec v, PetscInt* lo, PetscInt* hi) { *lo = 0; *hi = (PetscInt)v->a.size(); return 0; }
PetscErrorCode VecScatterCreate(Vec, IS ix, Vec, IS iy, VecScatter* sc) {
    *sc = new _p_VecScatter;
    (*sc)->from = ix->idx;
    (*sc)->to = iy->idx;
    return 0;
}
PetscErrorCode VecScatterCreateToAll(Vec x, VecScatter* sc, Vec* out) {
    *sc = new _p_VecScatter;
    (*sc)->to_all = true;
    VecDuplicate(x, out);
    return 0;
}
PetscErrorCode VecScatterBegin(VecScatter sc, Vec x, Vec y, InsertMode mode, ScatterMode smode) {
    if (sc->to_all) {
        if (smode == SCATTER_FORWARD) y->a = x->a; else x->a = y->a;
        return 0;
    }
    const auto& from = smode == SCATTER_FORWARD ? sc->from : sc->to;
    const auto& to = smode == SCATTER_FORWARD ? sc->to : sc->from;
    Vec src = smode == SCATTER_FORWARD ? x : y;
    Vec dst = smode == SCATTER_FORWARD ? y : x;
    for (size_t k = 0; k < from.size(); ++k) {
        if (mode == ADD_VALUES) dst->a[to[k]] += src->a[from[k]];
        else dst->a[to[k]] = src->a[from[k]];
    }
    return 0;
}
PetscErrorCode VecScatterEnd(VecScatter, Vec, Vec, InsertMode, ScatterMode) { return 0; }
PetscErrorCode VecScatterDestroy(VecScatter* sc) { if (sc && *sc) { delete *sc; *sc = nullptr; } return 0; }

// ---- IS ---------------------------------------------------------------
PetscErrorCode ISCreateGeneral(MPI_Comm, PetscInt n, const PetscInt idx[], PetscCopyMode, IS* is) {
    *is = new _p_IS;
    (*is)->idx.assign(idx, idx + (n > 0 ? n : 0));
    return 0;
}
PetscErrorCode ISDestroy(IS* is) { if (is && *is) { delete *is; *is = nullptr; } return 0; }

// ---- Mat --------------------------------------------------------------
PetscErrorCode MatCreate(MPI_Comm, Mat* A) { *A = new _p_Mat; return 0; }
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N) {
    A->ensure_sparse(m >= 0 ? m : M, n >= 0 ? n : N);
    return 0;
}
PetscErrorCode MatSetType(Mat A, MatType t) { A->dense = (std::string(t).find("dense") != std::string::npos); return 0; }
PetscErrorCode MatSetFromOptions(Mat) { return 0; }
PetscErrorCode MatMPIAIJSetPreallocation(Mat A, PetscInt, const PetscInt d_nnz[], PetscInt, const PetscInt o_nnz[]) {
    for (int i = 0; i < A->m; ++i) {
        int r = (d_nnz ? d_nnz[i] : 0) + (o_nnz ? o_nnz[i] : 0);
        A->cols[i].reserve(r);
        A->vals[i].reserve(r);
    }
    return 0;
}
PetscErrorCode MatSeqAIJSetPreallocation(Mat A, PetscInt, const PetscInt nnz[]) {
    for (int i = 0; i < A->m && nnz; ++i) { A->cols[i].reserve(nnz[i]); A->vals[i].reserve(nnz[i]); }
    return 0;
}
PetscErrorCode MatCreateSeqAIJ(MPI_Comm c, PetscInt m, PetscInt n, PetscInt nz, const PetscInt nnz[], Mat* A) {
    MatCreate(c, A);
    (*A)->ensure_sparse(m, n);
    return MatSeqAIJSetPreallocation(*A, nz, nnz);
}
PetscErrorCode MatCreateSeqDense(MPI_Comm c, PetscInt m, PetscInt n, PetscScalar* data, Mat* A) {
    MatCreate(c, A);
    (*A)->m = m; (*A)->n = n; (*A)->dense = true;
    (*A)->dd.assign((size_t)m * n, 0.0);
    if (data) std::copy(data, data + (size_t)m * n, (*A)->dd.begin());
    return 0;
}
PetscErrorCode MatCreateDense(MPI_Comm c, PetscInt m, PetscInt n, PetscInt M, PetscInt N, PetscScalar* data, Mat* A) {
    return MatCreateSeqDense(c, m >= 0 ? m : M, n >= 0 ? n : N, data, A);
}
PetscErrorCode MatSetUp(Mat) { return 0; }
PetscErrorCode MatSetOption(Mat, MatOption, PetscBool) { return 0; }
PetscErrorCode MatSetBlockSize(Mat, PetscInt) { return 0; }
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode) {
    if (i < 0 || j < 0) return 0;
    if (i >= A->m || j >= A->n) shim_fail("MatSetValue out of range");
    ++A->version;
    if (A->dense) {
        double& e = A->dd[(size_t)j * A->m + i];
        if (mode == ADD_VALUES) e += v; else e = v;
        return 0;
    }
    auto& cs = A->cols[i];
    auto& vs = A->vals[i];
    auto it = std::lower_bound(cs.begin(), cs.end(), j);
    size_t k = (size_t)(it - cs.begin());
    if (it == cs.end() || *it != j) {
        cs.insert(it, j);
        vs.insert(vs.begin() + k, 0.0);
    }
    if (mode == ADD_VALUES) vs[k] += v; else vs[k] = v;
    return 0;
}
PetscErrorCode MatSetValues(Mat A, PetscInt m, const PetscInt im[], PetscInt n, const PetscInt in[], const PetscScalar v[], InsertMode mode) {
    for (PetscInt a = 0; a < m; ++a)
        for (PetscInt b = 0; b < n; ++b) MatSetValue(A, im[a], in[b], v[(size_t)a * n + b], mode);
    return 0;
}
PetscErrorCode MatGetValues(Mat A, PetscInt m, const PetscInt im[], PetscInt n, const PetscInt in[], PetscScalar v[]) {
    for (PetscInt a = 0; a < m; ++a)
        for (PetscInt b = 0; b < n; ++b) {
            double val = 0.0;
            if (A->dense) val = A->dd[(size_t)in[b] * A->m + im[a]];
            else {
                const auto& cs = A->cols[im[a]];
                auto it = std::lower_bound(cs.begin(), cs.end(), in[b]);
                if (it != cs.end() && *it == in[b]) val = A->vals[im[a]][it - cs.begin()];
            }
            v[(size_t)a * n + b] = val;
        }
    return 0;
}
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType) { return 0; }
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType) { ++A->version; return 0; }
PetscErrorCode MatZeroEntries(Mat A) {
    ++A->version;
    if (A->dense) std::fill(A->dd.begin(), A->dd.end(), 0.0);
    else for (auto& vs : A->vals) std::fill(vs.begin(), vs.end(), 0.0);
    return 0;
}
PetscErrorCode MatDestroy(Mat* A) {
    if (A && *A) { delete (*A)->fac; delete *A; *A = nullptr; }
    return 0;
}
static void spmv(Mat A, const std::vector<double>& x, std::vector<double>& y, bool add) {
    if (!add) y.assign(A->m, 0.0);
    if (A->dense) {
        for (int j = 0; j < A->n; ++j)
            for (int i = 0; i < A->m; ++i) y[i] += A->dd[(size_t)j * A->m + i] * x[j];
        return;
    }
    for (int i = 0; i < A->m; ++i) {
        double s = 0.0;
        const auto& cs = A->cols[i];
        const auto& vs = A->vals[i];
        for (size_t k = 0; k < cs.size(); ++k) s += vs[k] * x[cs[k]];
        y[i] += s;
    }
}
PetscErrorCode MatMult(Mat A, Vec x, Vec y) { spmv(A, x->a, y->a, false); return 0; }
PetscErrorCode MatMultAdd(Mat A, Vec x, Vec y, Vec z) {
    std::vector<double> t = y->a;
    spmv(A, x->a, t, true);
    z->a = t;
    return 0;
}
PetscErrorCode MatMultTranspose(Mat A, Vec x, Vec y) {
    y->a.assign(A->n, 0.0);
    if (A->dense) {
        for (int j = 0; j < A->n; ++j)
            for (int i = 0; i < A->m; ++i) y->a[j] += A->dd[(size_t)j * A->m + i] * x->a[i];
        return 0;
    }
    for (int i = 0; i < A->m; ++i) {
        const auto& cs = A->cols[i];
        const auto& vs = A->vals[i];
        for (size_t k = 0; k < cs.size(); ++k) y->a[cs[k]] += vs[k] * x->a[i];
    }
    return 0;
}
PetscErrorCode MatGetSize(Mat A, PetscInt* m, PetscInt* n) { if (m) *m = A->m; if (n) *n = A->n; return 0; }
PetscErrorCode MatGetLocalSize(Mat A, PetscInt* m, PetscInt* n) { return MatGetSize(A, m, n); }
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt* lo, PetscInt* hi) { *lo = 0; *hi = A->m; return 0; }
PetscErrorCode MatGetOwnershipRangeColumn(Mat A, PetscInt* lo, PetscInt* hi) { *lo = 0; *hi = A->n; return 0; }
PetscErrorCode MatGetColumnVector(Mat A, Vec v, PetscInt col) {
    v->a.assign(A->m, 0.0);
    if (A->dense) { for (int i = 0; i < A->m; ++i) v->a[i] = A->dd[(size_t)col * A->m + i]; return 0; }
    for (int i = 0; i < A->m; ++i) {
        const auto& cs = A->cols[i];
        auto it = std::lower_bound(cs.begin(), cs.end(), col);
        if (it != cs.end() && *it == col) v->a[i] = A->vals[i][it - cs.begin()];
    }
    return 0;
}
PetscErrorCode MatGetOrdering(Mat, MatOrderingType, IS* r, IS* c) { *r = new _p_IS; *c = new _p_IS; return 0; }
PetscErrorCode MatGetFactor(Mat A, MatSolverPackage, MatFactorType, Mat* F) {
    *F = new _p_Mat;
    (*F)->factor_of = A;
    (*F)->m = A->m; (*F)->n = A->n;
    return 0;
}
PetscErrorCode MatCholeskyFactorSymbolic(Mat, Mat, IS, const MatFactorInfo*) { return 0; }
PetscErrorCode MatCholeskyFactorNumeric(Mat F, Mat A, const MatFactorInfo*) {
    delete F->fac;
    F->fac = new SkylineLDLT;
    F->fac->factor(A);
    return 0;
}
PetscErrorCode MatMatSolve(Mat F, Mat B, Mat X) {
    if (!F->fac || !B->dense || !X->dense) shim_fail("MatMatSolve");
    for (int j = 0; j < B->n; ++j) F->fac->solve(&B->dd[(size_t)j * B->m], &X->dd[(size_t)j * X->m]);
    return 0;
}
PetscErrorCode MatTranspose(Mat, int, Mat*) { shim_fail("MatTranspose"); }

// ---- KSP --------------------------------------------------------------
PetscErrorCode KSPCreate(MPI_Comm, KSP* ksp) { *ksp = new _p_KSP; return 0; }
PetscErrorCode KSPDestroy(KSP* ksp) { if (ksp && *ksp) { delete *ksp; *ksp = nullptr; } return 0; }
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat) { ksp->A = A; ksp->fac_version = -1; return 0; }
PetscErrorCode KSPGetPC(KSP ksp, PC* pc) { *pc = &ksp->pc; return 0; }
PetscErrorCode KSPSetType(KSP ksp, KSPType t) { ksp->type = t; return 0; }
PetscErrorCode KSPCGSetType(KSP, KSPCGType) { return 0; }
PetscErrorCode KSPSetTolerances(KSP, PetscReal, PetscReal, PetscReal, PetscInt) { return 0; }
PetscErrorCode KSPSetFromOptions(KSP) { return 0; }
PetscErrorCode KSPSetUp(KSP) { return 0; }
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x) {
    if (!ksp->A) shim_fail("KSPSolve without operator");
    const double t0 = now_s();
    if (ksp->fac_version != ksp->A->version || ksp->fac_mat != ksp->A || !ksp->fac.ok) {
        ksp->fac.factor(ksp->A);
        ksp->fac_version = ksp->A->version;
        ksp->fac_mat = ksp->A;
    }
    x->a.resize(b->a.size());
    ksp->fac.solve(b->a.data(), x->a.data());
    g_ksp_seconds += now_s() - t0;
    ++g_ksp_solves;
    return 0;
}
PetscErrorCode KSPSolveTranspose(KSP ksp, Vec b, Vec x) { return KSPSolve(ksp, b, x); }
PetscErrorCode PCSetType(PC pc, PCType t) { pc->type = t; return 0; }
PetscErrorCode PCFactorSetMatSolverPackage(PC, MatSolverPackage) { return 0; }
PetscErrorCode PCHYPRESetType(PC, const char*) { return 0; }
PetscErrorCode PCSetCoordinates(PC, PetscInt, PetscInt, PetscReal*) { return 0; }

// ---- SNES -------------------------------------------------------------
// PETSc's SNES defaults are rtol = stol = 1e-8 (what the reference runs with:
// its SNESSetTolerances passes PETSC_DEFAULT, SolverNonlinearSNES.cpp:78).
// PGSHIM_SNES_RTOL / PGSHIM_SNES_STOL replace those defaults when set -- the
// stand-in for PETSc's -snes_rtol / -snes_stol options, used to record
// tightly converged reference trajectories for parity tests.
PetscErrorCode SNESCreate(MPI_Comm, SNES* s) {
    *s = new _p_SNES;
    if (const char* v = std::getenv("PGSHIM_SNES_RTOL")) (*s)->rtol = std::atof(v);
    if (const char* v = std::getenv("PGSHIM_SNES_STOL")) (*s)->stol = std::atof(v);
    return 0;
}
PetscErrorCode SNESDestroy(SNES* s) { if (s && *s) { delete *s; *s = nullptr; } return 0; }
PetscErrorCode SNESGetKSP(SNES s, KSP* ksp) { *ksp = &s->ksp; return 0; }
PetscErrorCode SNESSetType(SNES, SNESType) { return 0; }
PetscErrorCode SNESSetTolerances(SNES s, PetscReal atol, PetscReal rtol, PetscReal stol, PetscInt maxit, PetscInt maxf) {
    if (atol != PETSC_DEFAULT) s->atol = atol;
    if (rtol != PETSC_DEFAULT) s->rtol = rtol;
    if (stol != PETSC_DEFAULT) s->stol = stol;
    if (maxit != PETSC_DEFAULT) s->maxit = maxit;
    if (maxf != PETSC_DEFAULT) s->maxf = maxf;
    return 0;
}
PetscErrorCode SNESSetFunction(SNES s, Vec r, SNESFunctionFn f, void* ctx) { s->r = r; s->f = f; s->fctx = ctx; return 0; }
PetscErrorCode SNESSetJacobian(SNES s, Mat A, Mat, SNESJacobianFn f, void* ctx) { s->J = A; s->jac = f; s->jctx = ctx; return 0; }
PetscErrorCode SNESMonitorSet(SNES s, SNESMonitorFn f, void* ctx, void*) { s->mon = f; s->mctx = ctx; return 0; }

static double norm2(const std::vector<double>& a) {
    double s = 0.0;
    for (double e : a) s += e * e;
    return std::sqrt(s);
}

// Newton with a backtracking line search (sufficient-decrease parameter
// alpha = 1e-4, quadratic then cubic interpolation, minimum step 1e-12),
// following the documented behaviour of PETSc's SNESNEWTONLS with the "bt"
// line search.  Convergence: ||F|| < atol, ||F|| <= rtol*||F0||,
// ||step|| < stol*||x||; maxit exceeded is DIVERGED_MAX_IT.
PetscErrorCode SNESSolve(SNES s, Vec b, Vec x) {
    PetscErrorCode ierr;
    if (b) shim_fail("SNESSolve with a right-hand side");
    Vec F = s->r, Y, W, G;
    VecDuplicate(x, &Y); VecDuplicate(x, &W); VecDuplicate(x, &G);
    s->reason = SNES_CONVERGED_ITERATING;
    s->its = 0;
    int nf = 0;
    ierr = s->f(s, x, F, s->fctx); CHKERRQ(ierr); ++nf;
    double fnorm = norm2(F->a);
    s->fnorm = fnorm;
    if (s->mon) s->mon(s, 0, fnorm, s->mctx);
    if (fnorm != fnorm) { s->reason = SNES_DIVERGED_FNORM_NAN; goto done; }
    if (fnorm < s->atol) { s->reason = SNES_CONVERGED_FNORM_ABS; goto done; }
    {
        const double ttol = fnorm * s->rtol;
        for (int it = 0; it < s->maxit; ++it) {
            ierr = s->jac(s, x, s->J, s->J, s->jctx); CHKERRQ(ierr);
            KSPSetOperators(&s->ksp, s->J, s->J);
            ierr = KSPSolve(&s->ksp, F, Y); CHKERRQ(ierr);
            // initial slope of 0.5*||F||^2 along -Y is -(F, J Y)
            spmv(s->J, Y->a, W->a, false);
            double initslope = 0.0;
            for (size_t i = 0; i < F->a.size(); ++i) initslope += F->a[i] * W->a[i];
            initslope = -initslope;
            if (initslope > 0.0) initslope = -initslope;
            if (initslope == 0.0) initslope = -1.0;
            const double alpha = 1e-4, minlambda = 1e-12;
            double lambda = 1.0, lambdaprev = 1.0, gnormprev = 0.0, gnorm;
            auto trial = [&](double lam) -> PetscErrorCode {
                for (size_t i = 0; i < x->a.size(); ++i) W->a[i] = x->a[i] - lam * Y->a[i];
                PetscErrorCode e = s->f(s, W, G, s->fctx); ++nf;
                gnorm = norm2(G->a);
                return e;
            };
            ierr = trial(lambda); CHKERRQ(ierr);
            const double f2 = fnorm * fnorm;
            bool accepted = (0.5 * gnorm * gnorm <= 0.5 * f2 + lambda * alpha * initslope);
            int bt = 0;
            while (!accepted && gnorm == gnorm) {
                double lambdatemp;
                if (bt == 0) {
                    lambdatemp = -initslope / (gnorm * gnorm - f2 - 2.0 * initslope);
                } else {
                    const double t1 = 0.5 * (gnorm * gnorm - f2) - lambda * initslope;
                    const double t2 = 0.5 * (gnormprev * gnormprev - f2) - lambdaprev * initslope;
                    const double a = (t1 / (lambda * lambda) - t2 / (lambdaprev * lambdaprev)) / (lambda - lambdaprev);
                    const double bb = (-lambdaprev * t1 / (lambda * lambda) + lambda * t2 / (lambdaprev * lambdaprev)) / (lambda - lambdaprev);
                    if (a == 0.0) lambdatemp = -initslope / (2.0 * bb);
                    else {
                        const double disc = bb * bb - 3.0 * a * initslope;
                        lambdatemp = disc < 0.0 ? 0.5 * lambda : (-bb + std::sqrt(disc)) / (3.0 * a);
                    }
                }
                lambdaprev = lambda;
                gnormprev = gnorm;
                if (lambdatemp > 0.5 * lambda) lambdatemp = 0.5 * lambda;
                lambda = std::max(lambdatemp, 0.1 * lambda);
                if (lambda < minlambda) break;
                ierr = trial(lambda); CHKERRQ(ierr);
                accepted = (0.5 * gnorm * gnorm <= 0.5 * f2 + lambda * alpha * initslope);
                ++bt;
            }
            if (gnorm != gnorm) { s->reason = SNES_DIVERGED_FNORM_NAN; goto done; }
            if (!accepted) { s->reason = SNES_DIVERGED_LINE_SEARCH; goto done; }
            x->a = W->a;
            F->a = G->a;
            fnorm = gnorm;
            s->fnorm = fnorm;
            s->its = it + 1;
            ++g_snes_iterations;
            if (s->mon) s->mon(s, s->its, fnorm, s->mctx);
            const double ynorm = lambda * norm2(Y->a);
            const double xnorm = norm2(x->a);
            if (fnorm != fnorm) { s->reason = SNES_DIVERGED_FNORM_NAN; goto done; }
            if (fnorm < s->atol) { s->reason = SNES_CONVERGED_FNORM_ABS; goto done; }
            if (nf >= s->maxf) { s->reason = SNES_DIVERGED_FUNCTION_COUNT; goto done; }
            if (fnorm <= ttol) { s->reason = SNES_CONVERGED_FNORM_RELATIVE; goto done; }
            if (ynorm < s->stol * xnorm) { s->reason = SNES_CONVERGED_SNORM_RELATIVE; goto done; }
        }
        s->reason = SNES_DIVERGED_MAX_IT;
    }
done:
    if (g_snes_verbose) fprintf(stderr, "[pg-ref-shim] SNES its=%d fnorm=%.3e reason=%d\n", s->its, s->fnorm, (int)s->reason);
    VecDestroy(&Y); VecDestroy(&W); VecDestroy(&G);
    return 0;
}
PetscErrorCode SNESGetFunctionNorm(SNES s, PetscReal* norm) { *norm = s->fnorm; return 0; }
PetscErrorCode SNESGetConvergedReason(SNES s, SNESConvergedReason* r) { *r = s->reason; return 0; }
PetscErrorCode SNESGetIterationNumber(SNES s, PetscInt* its) { *its = s->its; return 0; }

// ---- introspection for the oracle driver -------------------------------
PetscInt pgshim_mat_rows(Mat A) { return A->m; }
PetscInt pgshim_mat_cols(Mat A) { return A->n; }
PetscInt pgshim_mat_row_nnz(Mat A, PetscInt row) { return A->dense ? A->n : (PetscInt)A->cols[row].size(); }
void pgshim_mat_row(Mat A, PetscInt row, PetscInt* cols, PetscScalar* vals) {
    if (A->dense) {
        for (int j = 0; j < A->n; ++j) { cols[j] = j; vals[j] = A->dd[(size_t)j * A->m + row]; }
        return;
    }
    std::copy(A->cols[row].begin(), A->cols[row].end(), cols);
    std::copy(A->vals[row].begin(), A->vals[row].end(), vals);
}
PetscInt pgshim_vec_size(Vec v) { return (PetscInt)v->a.size(); }
PetscScalar* pgshim_vec_data(Vec v) { return v->a.data(); }
double pgshim_ksp_seconds(void) { return g_ksp_seconds; }
long pgshim_ksp_solves(void) { return g_ksp_solves; }
long pgshim_snes_iterations(void) { return g_snes_iterations; }
void pgshim_set_snes_verbose(int v) { g_snes_verbose = v; }

}  // extern "C"

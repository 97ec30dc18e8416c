// petsc_stub.h -- stand-in for the few PETSc / MPI names that fr_sdg's hot-path
// headers use, so that those headers compile unmodified without PETSc.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref): it lets the reference's own residual,
// limiter and change-of-variables code run on the CPU as the checker of the
// restated oracle.  Only what that code needs is implemented, for ONE rank:
//   * DMDA 1D/2D with `dof` values per element, stencil width 1, periodic or
//     ghosted boundaries (a DM_BOUNDARY_GHOSTED ghost element stays zero, as in
//     a freshly created local vector);
//   * global/local vectors as plain arrays, DMGlobalToLocal with the periodic wrap;
//   * DMDAVecGetArrayDOF(Read): an array of element pointers indexed [j][i] (or
//     [i]) over the owned or ghosted range, like PETSc's.
// The options database, MPI and the TS/SNES names are inert: parse_options and
// is_rank_0 compile but are never reached by the checker.
#pragma once
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <vector>

typedef int    PetscErrorCode;
typedef double PetscReal;
typedef double PetscScalar;
typedef int    PetscInt;
typedef int    PetscMPIInt;
typedef int    PetscEnum;
typedef bool PetscBool;  // PETSc defines it as bool for C++ builds
#define PETSC_FALSE false
#define PETSC_TRUE true

#define PETSC_SUCCESS 0
#define PETSC_ERR_SUP 56
#define PetscFunctionBeginUser do { } while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x)                                                                              \
    do                                                                                            \
    {                                                                                             \
        PetscErrorCode ierr_stub_ = (x);                                                          \
        if (ierr_stub_) return ierr_stub_;                                                        \
    } while (0)
#define PetscCallVoid(x) do { (void)(x); } while (0)
#define SETERRQ(comm, code, ...) return (code)

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define PETSC_COMM_WORLD 0
#define MPIU_SUM 0
#define MPIU_REAL 0
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype, MPI_Op, int, MPI_Comm)
{
    std::memcpy(r, s, sizeof(double) * static_cast<size_t>(n));
    return 0;
}

// ---- options database (inert) ------------------------------------------
#define PetscOptionsBegin(comm, prefix, title, sec) do { } while (0)
#define PetscOptionsEnd() do { } while (0)
inline PetscErrorCode PetscOptionsGetReal(void*, const char*, const char*, PetscReal*, PetscBool* set)
{
    if (set) *set = PETSC_FALSE;
    return 0;
}
inline PetscErrorCode PetscOptionsGetInt(void*, const char*, const char*, PetscInt*, PetscBool* set)
{
    if (set) *set = PETSC_FALSE;
    return 0;
}
inline PetscErrorCode PetscOptionsGetBool(void*, const char*, const char*, PetscBool*, PetscBool* set)
{
    if (set) *set = PETSC_FALSE;
    return 0;
}
inline PetscErrorCode PetscOptionsEnum(const char*, const char*, const char*, const char* const*, PetscEnum,
                                       PetscEnum*, PetscBool* set)
{
    if (set) *set = PETSC_FALSE;
    return 0;
}
inline PetscErrorCode PetscOptionsGetEnum(void*, const char*, const char*, const char* const*, PetscEnum*,
                                          PetscBool* set)
{
    if (set) *set = PETSC_FALSE;
    return 0;
}
inline PetscErrorCode PetscInitialize(int*, char***, const char*, const char*) { return 0; }
inline PetscErrorCode PetscFinalize() { return 0; }
template <class... A> inline PetscErrorCode PetscPrintf(MPI_Comm, const char*, A...) { return 0; }

// ---- solver handles (opaque, never used by the checker) -------------------
typedef struct StubTS_*   TS;
typedef struct StubSNES_* SNES;
typedef struct StubMat_*  Mat;
typedef struct StubKSP_*  KSP;
typedef struct StubPC_*   PC;
typedef const char*       TSType;
typedef const char*       PCType;
#define TSBDF "bdf"
#define TSTHETA "theta"
#define TSALPHA "alpha"
#define TSBEULER "beuler"
#define TSCN "cn"
#define TSARKIMEX "arkimex"
#define TSROSW "rosw"
inline PetscErrorCode TSGetType(TS, TSType* t) { *t = "ssp"; return 0; }

// ---- DMDA ------------------------------------------------------------------
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_PERIODIC } DMBoundaryType;
typedef enum { INSERT_VALUES, ADD_VALUES } InsertMode;

struct StubVec_;
struct StubDM_
{
    int dim{2};
    int nx{1}, ny{1}, dof{1};
    bool per_x{false}, per_y{false};
    // local vectors handed out by DMGetLocalVector and kept for reuse, like PETSc's
    // pool (a reused vector keeps its ghost entries, which nothing writes at a
    // ghosted boundary, so they stay zero)
    std::vector<std::pair<StubVec_*, bool>> pool;
    ~StubDM_();
};
typedef StubDM_* DM;

// A vector is a view of `n` doubles at `ptr`: storage it owns (the DM's local
// vectors) or memory of the caller (global vectors wrap the caller's arrays).
struct StubVec_
{
    std::vector<double> own;
    double* ptr{nullptr};
    size_t  n{0};
    bool    local{false};
    // pointer tables handed out by DMDAVecGetArrayDOF(Read)
    std::vector<double*>  rows1;
    std::vector<double**> rows2;
};
typedef StubVec_* Vec;

inline StubDM_::~StubDM_()
{
    for (auto& v : pool) delete v.first;
}

// Element ranges: owned [0, n), ghosted [-1, n+1) along every axis (stencil width 1).
inline int stub_ghost_w(const StubDM_* d) { return d->nx + 2; }
inline int stub_ghost_h(const StubDM_* d) { return d->dim == 2 ? d->ny + 2 : 1; }
inline size_t stub_local_size(const StubDM_* d) { return size_t(stub_ghost_w(d)) * stub_ghost_h(d) * d->dof; }

inline PetscErrorCode DMDAGetCorners(DM da, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n,
                                     PetscInt* p)
{
    if (x) *x = 0;
    if (y) *y = 0;
    if (z) *z = 0;
    if (m) *m = da->nx;
    if (n) *n = da->ny;
    if (p) *p = 1;
    return 0;
}
inline PetscErrorCode DMDAGetGhostCorners(DM da, PetscInt* x, PetscInt* y, PetscInt* z, PetscInt* m, PetscInt* n,
                                          PetscInt* p)
{
    if (x) *x = -1;
    if (y) *y = -1;
    if (z) *z = 0;
    if (m) *m = da->nx + 2;
    if (n) *n = da->ny + 2;
    if (p) *p = 1;
    return 0;
}

inline PetscErrorCode DMGetLocalVector(DM da, Vec* v)
{
    for (auto& e : da->pool)
        if (!e.second)
        {
            e.second = true;
            *v = e.first;
            return 0;
        }
    auto* lv  = new StubVec_;
    lv->local = true;
    lv->own.assign(stub_local_size(da), 0.0);
    lv->ptr = lv->own.data();
    lv->n   = lv->own.size();
    da->pool.emplace_back(lv, true);
    *v = lv;
    return 0;
}
inline PetscErrorCode DMRestoreLocalVector(DM da, Vec* v)
{
    for (auto& e : da->pool)
        if (e.first == *v) e.second = false;
    *v = nullptr;
    return 0;
}

// Local vector offset of ghosted element (i, j), i in [-1, nx], j in [-1, ny].
inline size_t stub_local_off(const StubDM_* d, int i, int j)
{
    const int jj = d->dim == 2 ? j + 1 : 0;
    return (size_t(jj) * stub_ghost_w(d) + size_t(i + 1)) * d->dof;
}

// The ghost scatter of rows [j_lo, j_hi] (inclusive; 2D rows may reach -1 and ny,
// 1D uses row 0) from the global array g into the local array l: owned elements
// and the periodic wrap; ghosts at a ghosted boundary are left as they are.
inline void stub_scatter_rows(const StubDM_* da, const double* g, double* l, int j_lo, int j_hi)
{
    for (int j = j_lo; j <= j_hi; ++j)
        for (int i = -1; i <= da->nx; ++i)
        {
            int si = i, sj = j;
            bool ok = true;
            if (si < 0 || si >= da->nx)
            {
                if (!da->per_x) ok = false;
                si = (si + da->nx) % da->nx;
            }
            if (da->dim == 2 && (sj < 0 || sj >= da->ny))
            {
                if (!da->per_y) ok = false;
                sj = (sj + da->ny) % da->ny;
            }
            if (!ok) continue;
            const size_t go = (size_t(da->dim == 2 ? sj : 0) * da->nx + size_t(si)) * da->dof;
            std::memcpy(l + stub_local_off(da, i, j), g + go, sizeof(double) * da->dof);
        }
}

inline PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec) { return 0; }
inline PetscErrorCode DMGlobalToLocalEnd(DM da, Vec g, InsertMode, Vec l)
{
    if (da->dim == 2) stub_scatter_rows(da, g->ptr, l->ptr, -1, da->ny);
    else stub_scatter_rows(da, g->ptr, l->ptr, 0, 0);
    return 0;
}

inline PetscErrorCode DMDAVecGetArrayDOF(DM da, Vec v, void* arr)
{
    if (da->dim == 1)
    {
        const int lo = v->local ? -1 : 0, cnt = v->local ? da->nx + 2 : da->nx;
        v->rows1.assign(size_t(cnt), nullptr);
        for (int i = 0; i < cnt; ++i) v->rows1[size_t(i)] = v->ptr + size_t(i) * da->dof;
        *static_cast<double***>(arr) = v->rows1.data() - lo;
        return 0;
    }
    const int lo = v->local ? -1 : 0;
    const int w = v->local ? da->nx + 2 : da->nx, h = v->local ? da->ny + 2 : da->ny;
    v->rows1.assign(size_t(w) * h, nullptr);
    v->rows2.assign(size_t(h), nullptr);
    for (int j = 0; j < h; ++j)
    {
        for (int i = 0; i < w; ++i) v->rows1[size_t(j) * w + i] = v->ptr + (size_t(j) * w + i) * da->dof;
        v->rows2[size_t(j)] = v->rows1.data() + size_t(j) * w - lo;
    }
    *static_cast<double****>(arr) = v->rows2.data() - lo;
    return 0;
}
inline PetscErrorCode DMDAVecGetArrayDOFRead(DM da, Vec v, void* arr) { return DMDAVecGetArrayDOF(da, v, arr); }
inline PetscErrorCode DMDAVecRestoreArrayDOF(DM, Vec, void*) { return 0; }
inline PetscErrorCode DMDAVecRestoreArrayDOFRead(DM, Vec, void*) { return 0; }

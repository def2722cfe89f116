/*
 * mgp_oracle.c -- CPU restatement of the reference multigrid hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine is compared
 * against; it is loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
 * leg, and by nothing in the product path.
 *
 * It restates, in plain sequential C and FP64, the operation sequence of the reference
 * eljens/multigrid-poisson (Poisson::PoissonSolver<double,R,TrilinearInterpolation,S>),
 * on arrays in the reference's own halo-padded layout (include/array.h:20-30,70-77):
 *     idx(i,j,k) = (i+halo.west)*S0 + (j+halo.south)*S1 + (k+halo.bottom),
 *     S0 = ny_p*nz_p, S1 = nz_p, k (z) unit-stride.
 * Every arithmetic expression keeps the reference's operand order, so with no FMA
 * contraction (-ffp-contract=off) results are bit-identical to the reference's own CPU
 * build; tests/test_oracle_pin.py pins this against the reference run through
 * oracle/ref_harness.cpp.  Red-black Gauss-Seidel follows the reference's colour rule
 * (parity of the padded linear index) in the reference's sequential i,j,k order, i.e. what
 * its OpenMP build computes on one thread.
 *
 * Build: gcc -O2 -std=c11 -ffp-contract=off -fPIC -shared mgp_oracle.c -lm
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define ORC_MAX_LEVELS 16

/* Face order of the reference's Location_t (include/boundary.h:12). */
enum { NORTH = 0, SOUTH, EAST, WEST, TOP, BOTTOM };
enum { ORC_D = 0, ORC_N = 1 };
enum { ORC_INJECTION = 0, ORC_FULLWEIGHTING = 1 };
enum { ORC_JACOBI = 0, ORC_GAUSSSEIDEL = 1 };
enum { ORC_U = 0, ORC_UPREV = 1, ORC_F = 2, ORC_R = 3 };

typedef struct {
    long shape[3];
    long pad[3];       /* halo-padded extents */
    long stride[3];
    long size;
    long hw, he, hs, hn, hb, ht; /* halo widths west/east/south/north/bottom/top */
    double h;
    long face_shape[6][3];
} orc_level;

typedef struct {
    int levels;
    int restriction, relaxation;
    int face_type[6];  /* resolved boundary kinds (Domain ctor, include/domain.h:125-192) */
    orc_level lv[ORC_MAX_LEVELS];
    double *u[ORC_MAX_LEVELS], *uprev[ORC_MAX_LEVELS], *f[ORC_MAX_LEVELS], *r[ORC_MAX_LEVELS];
    double *g[ORC_MAX_LEVELS][6];
    int gs_alternate; /* GaussSeidel::alternate (include/gaussseidel.h:18) */
    double origin[3];
} orc_solver;

static inline long IDX(const orc_level* L, long i, long j, long k) {
    return (i + L->hw) * L->stride[0] + (j + L->hs) * L->stride[1] + (k + L->hb);
}
/* Face arrays have no halo: strides {ny*nz, nz, 1} (include/array.h:65-68). */
static inline long FIDX(const long* fs, long i, long j, long k) { return i * fs[1] * fs[2] + j * fs[2] + k; }

/* ------------------------------------------------------------------------------------ */
/* Level geometry: DomainSettings(l) (src/domainsettings.cpp:12-29) and the halo widths of
 * Domain's constructor (include/domain.h:102-108), single device. */
int orc_create(const long dims[3], int levels, double h, const int bc_req[6], int restriction,
               int relaxation, int strict_bc, orc_solver** out) {
    if (levels < 1 || levels > ORC_MAX_LEVELS) return 1;
    orc_solver* S = (orc_solver*)calloc(1, sizeof(orc_solver));
    S->levels = levels;
    S->restriction = restriction;
    S->relaxation = relaxation;
    S->gs_alternate = 1;
    for (int fc = 0; fc < 6; fc++) S->face_type[fc] = bc_req[fc];
    if (!strict_bc) {
        /* north/south are always Dirichlet (domain.h:191-192); bottom always Dirichlet
         * (domain.h:140-145). */
        S->face_type[NORTH] = ORC_D;
        S->face_type[SOUTH] = ORC_D;
        S->face_type[BOTTOM] = ORC_D;
    }
    for (int l = 0; l < levels; l++) {
        orc_level* L = &S->lv[l];
        for (int d = 0; d < 3; d++) {
            long n = l > 0 ? (dims[d] >> l) + 1 : dims[d];
            if (l > 0 && (((n - 1) << l) + 1) != dims[d]) {
                free(S);
                return 2; /* std::invalid_argument in the reference */
            }
            L->shape[d] = n;
        }
        L->h = h * (double)(1L << l);
        /* halo widths follow the REQUESTED types */
        L->he = bc_req[EAST] != ORC_D;
        L->hw = bc_req[WEST] != ORC_D;
        L->hn = bc_req[NORTH] != ORC_D;
        L->hs = bc_req[SOUTH] != ORC_D;
        L->ht = bc_req[TOP] != ORC_D;
        L->hb = bc_req[BOTTOM] != ORC_D;
        L->pad[0] = L->shape[0] + L->he + L->hw;
        L->pad[1] = L->shape[1] + L->hn + L->hs;
        L->pad[2] = L->shape[2] + L->ht + L->hb;
        L->stride[0] = L->pad[1] * L->pad[2];
        L->stride[1] = L->pad[2];
        L->stride[2] = 1;
        L->size = L->pad[0] * L->pad[1] * L->pad[2];
        long nx = L->shape[0], ny = L->shape[1], nz = L->shape[2];
        long fsh[6][3] = {{nx, 1, nz}, {nx, 1, nz}, {1, ny, nz}, {1, ny, nz}, {nx, ny, 1}, {nx, ny, 1}};
        memcpy(L->face_shape, fsh, sizeof(fsh));
        S->u[l] = (double*)calloc(L->size, sizeof(double));
        S->uprev[l] = relaxation == ORC_JACOBI ? (double*)calloc(L->size, sizeof(double)) : S->u[l];
        S->f[l] = (double*)calloc(L->size, sizeof(double));
        S->r[l] = (double*)calloc(L->size, sizeof(double));
        for (int fc = 0; fc < 6; fc++)
            S->g[l][fc] = (double*)calloc(fsh[fc][0] * fsh[fc][1] * fsh[fc][2], sizeof(double));
    }
    *out = S;
    return 0;
}

void orc_destroy(orc_solver* S) {
    if (!S) return;
    for (int l = 0; l < S->levels; l++) {
        if (S->uprev[l] != S->u[l]) free(S->uprev[l]);
        free(S->u[l]);
        free(S->f[l]);
        free(S->r[l]);
        for (int fc = 0; fc < 6; fc++) free(S->g[l][fc]);
    }
    free(S);
}

/* meta: shape[3], pad[3], stride[3], size, halo[6] (e,w,n,s,t,b) */
void orc_level_meta(const orc_solver* S, int l, long* m) {
    const orc_level* L = &S->lv[l];
    for (int d = 0; d < 3; d++) {
        m[d] = L->shape[d];
        m[3 + d] = L->pad[d];
        m[6 + d] = L->stride[d];
    }
    m[9] = L->size;
    m[10] = L->he; m[11] = L->hw; m[12] = L->hn; m[13] = L->hs; m[14] = L->ht; m[15] = L->hb;
}
double orc_level_h(const orc_solver* S, int l) { return S->lv[l].h; }
int orc_face_type(const orc_solver* S, int fc) { return S->face_type[fc]; }

double* orc_field(orc_solver* S, int field, int l) {
    switch (field) {
        case ORC_U: return S->u[l];
        case ORC_UPREV: return S->uprev[l];
        case ORC_F: return S->f[l];
        default: return S->r[l];
    }
}
double* orc_face(orc_solver* S, int fc, int l) { return S->g[l][fc]; }

/* ------------------------------------------------------------------------------------ */
/* Problem plug-ins: same numbering as oracle/ref_harness.cpp. */
static const double kPi = 3.14159265358979323846;
static double p_u(int p, double x, double y, double z) {
    switch (p) {
        case 1: return sin(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return x * x * x * y * y * z;
        case 3: return cos(x * z * z) * sin(y * y * y);
        case 10: return sin(2.0 * kPi * x) * sin(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
static double p_f(int p, double x, double y, double z) {
    switch (p) {
        case 1: return -(3.0 * 3.0 + 5.3 * 5.3 + (-7.8) * (-7.8)) * sin(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return 2.0 * x * x * x * z + 6.0 * x * y * y * z;
        case 3:
            return ((-4.0 * x * x * z * z - 9.0 * y * y * y * y - z * z * z * z) * sin(y * y * y) +
                    6.0 * y * cos(y * y * y)) * cos(x * z * z) -
                   2.0 * x * sin(x * z * z) * sin(y * y * y);
        case 10: return -12.0 * kPi * kPi * sin(2.0 * kPi * x) * sin(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
static double p_dx(int p, double x, double y, double z) {
    switch (p) {
        case 1: return 3.0 * cos(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return 3.0 * x * x * y * y * z;
        case 3: return -z * z * sin(x * z * z) * sin(y * y * y);
        case 10: return 2.0 * kPi * cos(2.0 * kPi * x) * sin(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
static double p_dy(int p, double x, double y, double z) {
    switch (p) {
        case 1: return 5.3 * sin(3.0 * x) * cos(5.3 * y) * sin(-7.8 * z);
        case 2: return 2.0 * x * x * x * y * z;
        case 3: return 3.0 * cos(x * z * z) * y * y * cos(y * y * y);
        case 10: return 2.0 * kPi * sin(2.0 * kPi * x) * cos(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
static double p_dz(int p, double x, double y, double z) {
    switch (p) {
        case 1: return -7.8 * sin(3.0 * x) * sin(5.3 * y) * cos(-7.8 * z);
        case 2: return x * x * x * y * y;
        case 3: return -2 * x * z * sin(x * z * z) * sin(y * y * y);
        case 10: return 2.0 * kPi * sin(2.0 * kPi * x) * sin(2.0 * kPi * y) * cos(2.0 * kPi * z);
        default: return 0.0;
    }
}
double orc_problem_u(int p, double x, double y, double z) { return p_u(p, x, y, z); }

/* PoissonSolver::init (include/libpoisson.h:158-171): level 0 gets boundary data
 * (Boundary::init_by_fun, include/boundary.h:81-111; Dirichlet faces sample u, Neumann
 * faces the normal derivative, neumann.h:63-79) and f at every shape point
 * (Domain::init_f, include/domain.h:328-342); everything else is zero. */
void orc_init_problem(orc_solver* S, int p, const double origin[3]) {
    for (int l = 0; l < S->levels; l++) {
        orc_level* L = &S->lv[l];
        memset(S->u[l], 0, L->size * sizeof(double));
        if (S->uprev[l] != S->u[l]) memset(S->uprev[l], 0, L->size * sizeof(double));
        memset(S->f[l], 0, L->size * sizeof(double));
        memset(S->r[l], 0, L->size * sizeof(double));
        for (int fc = 0; fc < 6; fc++) {
            long* fs = L->face_shape[fc];
            memset(S->g[l][fc], 0, fs[0] * fs[1] * fs[2] * sizeof(double));
        }
    }
    S->origin[0] = origin[0];
    S->origin[1] = origin[1];
    S->origin[2] = origin[2];
    orc_level* L = &S->lv[0];
    const double x0 = origin[0], y0 = origin[1], z0 = origin[2], h = L->h;
    for (int fc = 0; fc < 6; fc++) {
        double offx = 0, offy = 0, offz = 0;
        if (fc == TOP) offz = (double)(L->shape[2] - 1);
        if (fc == NORTH) offy = (double)(L->shape[1] - 1);
        if (fc == EAST) offx = (double)(L->shape[0] - 1);
        long* fs = L->face_shape[fc];
        for (long i = 0; i < fs[0]; i++)
            for (long j = 0; j < fs[1]; j++)
                for (long k = 0; k < fs[2]; k++) {
                    double x = x0 + (((double)i) + offx) * h;
                    double y = y0 + (((double)j) + offy) * h;
                    double z = z0 + (((double)k) + offz) * h;
                    double v;
                    if (S->face_type[fc] == ORC_D) v = p_u(p, x, y, z);
                    else if (fc == EAST || fc == WEST) v = p_dx(p, x, y, z);
                    else if (fc == NORTH || fc == SOUTH) v = p_dy(p, x, y, z);
                    else v = p_dz(p, x, y, z);
                    S->g[0][fc][FIDX(fs, i, j, k)] = v;
                }
    }
    for (long i = 0; i < L->shape[0]; i++)
        for (long j = 0; j < L->shape[1]; j++)
            for (long k = 0; k < L->shape[2]; k++)
                S->f[0][IDX(L, i, j, k)] = p_f(p, x0 + ((double)i) * h, y0 + ((double)j) * h, z0 + ((double)k) * h);
}

/* ------------------------------------------------------------------------------------ */
/* Dirichlet::write_to (include/dirichlet.h:50-93): copy the face array into the boundary
 * plane.  Neumann::write_to (include/neumann.h:63-131): ghost = sign*2h*g + u[mirror]. */
static void write_face(orc_solver* S, int l, int fc, double* ua) {
    orc_level* L = &S->lv[l];
    long nx = L->shape[0], ny = L->shape[1], nz = L->shape[2];
    long* fs = L->face_shape[fc];
    const double* g = S->g[l][fc];
    if (S->face_type[fc] == ORC_D) {
        long offx = 0, offy = 0, offz = 0;
        if (fc == TOP) offz = nz - 1;
        if (fc == NORTH) offy = ny - 1;
        if (fc == EAST) offx = nx - 1;
        for (long i = 0; i < fs[0]; i++)
            for (long j = 0; j < fs[1]; j++)
                for (long k = 0; k < fs[2]; k++) ua[IDX(L, i + offx, j + offy, k + offz)] = g[FIDX(fs, i, j, k)];
        return;
    }
    long offx = 0, offy = 0, offz = 0, ii = 0, jj = 0, kk = 0;
    double sign = 1.0;
    switch (fc) {
        case EAST: offx = nx; ii = -2; break;
        case WEST: offx = -1; ii = 2; sign = -1.0; break;
        case NORTH: offy = ny; jj = -2; break;
        case SOUTH: offy = -1; jj = 2; sign = -1.0; break;
        case TOP: offz = nz; kk = -2; break;
        default: offz = -1; kk = 2; sign = -1.0; break;
    }
    const double two_h = 2.0 * L->h;
    for (long i = 0; i < fs[0]; i++)
        for (long j = 0; j < fs[1]; j++)
            for (long k = 0; k < fs[2]; k++)
                ua[IDX(L, i + offx, j + offy, k + offz)] =
                    sign * two_h * g[FIDX(fs, i, j, k)] + ua[IDX(L, i + offx + ii, j + offy + jj, k + offz + kk)];
}

/* Domain::write_bc_to (include/domain.h:318-326), done for u and uprev at to_device. */
void orc_write_bc(orc_solver* S, int l) {
    static const int order[6] = {NORTH, SOUTH, EAST, WEST, TOP, BOTTOM};
    for (int t = 0; t < 6; t++) write_face(S, l, order[t], S->u[l]);
    if (S->uprev[l] != S->u[l])
        for (int t = 0; t < 6; t++) write_face(S, l, order[t], S->uprev[l]);
}

/* Boundary::update for every face in the order of include/relaxation.h:35-52 and
 * include/residual.h:353-358 (Dirichlet::update is a no-op, dirichlet.h:95-99). */
static void update_ghosts(orc_solver* S, int l, double* ua) {
    static const int order[6] = {EAST, WEST, NORTH, SOUTH, TOP, BOTTOM};
    for (int t = 0; t < 6; t++)
        if (S->face_type[order[t]] == ORC_N) write_face(S, l, order[t], ua);
}

/* Interior bounds from Boundary::is_non_eliminated (relaxation.h:78-83): Dirichlet planes
 * are excluded, Neumann planes included. */
static void bounds(const orc_solver* S, int l, long b[6]) {
    const orc_level* L = &S->lv[l];
    b[0] = S->face_type[WEST] == ORC_D;
    b[1] = L->shape[0] - (S->face_type[EAST] == ORC_D);
    b[2] = S->face_type[SOUTH] == ORC_D;
    b[3] = L->shape[1] - (S->face_type[NORTH] == ORC_D);
    b[4] = S->face_type[BOTTOM] == ORC_D;
    b[5] = L->shape[2] - (S->face_type[TOP] == ORC_D);
}

/* Jacobi::relaxation_kernel (include/jacobi.h:39-82). */
static void jacobi_kernel(orc_solver* S, int l, double omega) {
    orc_level* L = &S->lv[l];
    double* u = S->u[l];
    const double* v = S->uprev[l];
    const double* f = S->f[l];
    const double one_omega = 1.0 - omega;
    const double omega_sixth = omega / 6.0;
    const double hsq = L->h * L->h;
    const long s0 = L->stride[0], s1 = L->stride[1];
    long b[6];
    bounds(S, l, b);
    for (long i = b[0]; i < b[1]; i++)
        for (long j = b[2]; j < b[3]; j++)
            for (long k = b[4]; k < b[5]; k++) {
                long c = IDX(L, i, j, k);
                u[c] = one_omega * v[c];
                u[c] += omega_sixth * (v[c - s0] + v[c + s0] + v[c - s1] + v[c + s1] + v[c - 1] + v[c + 1] - hsq * f[c]);
            }
}

/* GaussSeidel::relaxation_kernel (include/gaussseidel.h:28-94): one colour per call, the
 * colour being the parity of the padded linear index; alternate flips after each call. */
static void gs_kernel(orc_solver* S, int l, double omega) {
    orc_level* L = &S->lv[l];
    double* u = S->u[l];
    const double* f = S->f[l];
    const double one_omega = 1.0 - omega;
    const double omega_sixth = omega / 6.0;
    const double hsq = L->h * L->h;
    const long s0 = L->stride[0], s1 = L->stride[1];
    const long colour = S->gs_alternate ? 0 : 1;
    long b[6];
    bounds(S, l, b);
    for (long i = b[0]; i < b[1]; i++)
        for (long j = b[2]; j < b[3]; j++)
            for (long k = b[4]; k < b[5]; k++) {
                long c = IDX(L, i, j, k);
                if (c % 2 == colour)
                    u[c] = one_omega * u[c] +
                           omega_sixth * (u[c - s0] + u[c + s0] + u[c - s1] + u[c + s1] + u[c - 1] + u[c + 1] - hsq * f[c]);
            }
    S->gs_alternate = !S->gs_alternate;
}

/* Relaxation::relax (include/relaxation.h:19-94): smoothing_multiplier()*nsmooth
 * half-sweeps; Jacobi swaps u/uprev first (domain.h:311-316) and refreshes the ghosts of
 * the source (update(..., previous=true)). */
void orc_relax(orc_solver* S, int l, double omega, long nsmooth) {
    int mult = S->relaxation == ORC_GAUSSSEIDEL ? 2 : 1;
    for (long s = 0; s < mult * nsmooth; s++) {
        if (S->relaxation == ORC_JACOBI) {
            double* t = S->u[l];
            S->u[l] = S->uprev[l];
            S->uprev[l] = t;
            update_ghosts(S, l, S->uprev[l]);
            jacobi_kernel(S, l, omega);
        } else {
            update_ghosts(S, l, S->u[l]);
            gs_kernel(S, l, omega);
        }
    }
}

/* One red-black half-sweep of the given colour (the parity of the padded linear index), ghosts
 * refreshed first as orc_relax does; the alternate flag is left as it was.  The decomposed
 * solve orders the colours itself and exchanges halo planes between them. */
void orc_relax_colour(orc_solver* S, int l, double omega, int colour) {
    const int keep = S->gs_alternate;
    S->gs_alternate = colour == 0;
    update_ghosts(S, l, S->u[l]);
    gs_kernel(S, l, omega);
    S->gs_alternate = keep;
}

/* residual<T> (include/residual.h:17-81). */
void orc_residual(orc_solver* S, int l) {
    orc_level* L = &S->lv[l];
    update_ghosts(S, l, S->u[l]);
    const double* u = S->u[l];
    const double* f = S->f[l];
    double* r = S->r[l];
    const double hsq = L->h * L->h;
    const long s0 = L->stride[0], s1 = L->stride[1];
    long b[6];
    bounds(S, l, b);
    for (long i = b[0]; i < b[1]; i++)
        for (long j = b[2]; j < b[3]; j++)
            for (long k = b[4]; k < b[5]; k++) {
                long c = IDX(L, i, j, k);
                r[c] = f[c] - (u[c - s0] + u[c + s0] + u[c - s1] + u[c + s1] + u[c - 1] + u[c + 1] - 6.0 * u[c]) / hsq;
            }
}

/* Generic restriction between two arrays described by (shape, halo-aware index):
 * Injection::restrict_to (include/injection.h:29-67) and FullWeighting::restrict_to with
 * index clamping (include/fullweighting.h:37-122). */
typedef struct {
    const long* shape;
    long stride0, stride1, off; /* linear = i*stride0 + j*stride1 + k + off */
} view_t;
static inline long VI(const view_t* v, long i, long j, long k) { return i * v->stride0 + j * v->stride1 + k + v->off; }
static inline long lmin(long a, long b) { return a < b ? a : b; }
static inline long lmax(long a, long b) { return a > b ? a : b; }

static void restrict_view(int kind, const double* in, const view_t* vi, double* out, const view_t* vo) {
    const long* is = vi->shape;
    const long* os = vo->shape;
    for (long i = 0; i < os[0]; i++)
        for (long j = 0; j < os[1]; j++)
            for (long k = 0; k < os[2]; k++) {
                if (kind == ORC_INJECTION) {
                    out[VI(vo, i, j, k)] = in[VI(vi, 2 * i, 2 * j, 2 * k)];
                    continue;
                }
                long ii = lmin(is[0] - 1, 2 * i), jj = lmin(is[1] - 1, 2 * j), kk = lmin(is[2] - 1, 2 * k);
                long im = lmax(0, ii - 1), ip = lmin(is[0] - 1, ii + 1);
                long jm = lmax(0, jj - 1), jp = lmin(is[1] - 1, jj + 1);
                long km = lmax(0, kk - 1), kp = lmin(is[2] - 1, kk + 1);
                double t = 1.0 * in[VI(vi, im, jm, km)] + 2.0 * in[VI(vi, im, jj, km)] + 1.0 * in[VI(vi, im, jp, km)] +
                           2.0 * in[VI(vi, ii, jm, km)] + 4.0 * in[VI(vi, ii, jj, km)] + 2.0 * in[VI(vi, ii, jp, km)] +
                           1.0 * in[VI(vi, ip, jm, km)] + 2.0 * in[VI(vi, ip, jj, km)] + 1.0 * in[VI(vi, ip, jp, km)];
                t += 2.0 * in[VI(vi, im, jm, kk)] + 4.0 * in[VI(vi, im, jj, kk)] + 2.0 * in[VI(vi, im, jp, kk)] +
                     4.0 * in[VI(vi, ii, jm, kk)] + 8.0 * in[VI(vi, ii, jj, kk)] + 4.0 * in[VI(vi, ii, jp, kk)] +
                     2.0 * in[VI(vi, ip, jm, kk)] + 4.0 * in[VI(vi, ip, jj, kk)] + 2.0 * in[VI(vi, ip, jp, kk)];
                t += 1.0 * in[VI(vi, im, jm, kp)] + 2.0 * in[VI(vi, im, jj, kp)] + 1.0 * in[VI(vi, im, jp, kp)] +
                     2.0 * in[VI(vi, ii, jm, kp)] + 4.0 * in[VI(vi, ii, jj, kp)] + 2.0 * in[VI(vi, ii, jp, kp)] +
                     1.0 * in[VI(vi, ip, jm, kp)] + 2.0 * in[VI(vi, ip, jj, kp)] + 1.0 * in[VI(vi, ip, jp, kp)];
                out[VI(vo, i, j, k)] = t / 64.0;
            }
}

static view_t level_view(const orc_level* L) {
    view_t v = {L->shape, L->stride[0], L->stride[1], L->hw * L->stride[0] + L->hs * L->stride[1] + L->hb};
    return v;
}
static view_t face_view(const long* fs) {
    view_t v = {fs, fs[1] * fs[2], fs[2], 0};
    return v;
}

/* restriction.restrict_to(r_l, f_{l+1}) (include/vcycle.h:43-46). */
void orc_restrict(orc_solver* S, int l) {
    view_t vi = level_view(&S->lv[l]), vo = level_view(&S->lv[l + 1]);
    restrict_view(S->restriction, S->r[l], &vi, S->f[l + 1], &vo);
}

/* DeviceArray::init_zero of u_{l+1} (include/devicearray.h:132-159): the padded array. */
void orc_zero_u(orc_solver* S, int l) { memset(S->u[l], 0, S->lv[l].size * sizeof(double)); }

/* The six Boundary::restrict_to calls level l -> l+1 (include/vcycle.h:52-75):
 * Dirichlet: coarse g = 0 (dirichlet.h:101-107).  Neumann (neumann.h:146-252): coarse g =
 * R(fine g) minus a one-sided second-order normal derivative of the fine u, divided by
 * the fine h. */
void orc_restrict_bc(orc_solver* S, int l) {
    static const int order[6] = {NORTH, SOUTH, EAST, WEST, TOP, BOTTOM};
    orc_level* F = &S->lv[l];
    orc_level* C = &S->lv[l + 1];
    for (int t = 0; t < 6; t++) {
        int fc = order[t];
        long* cs = C->face_shape[fc];
        double* gc = S->g[l + 1][fc];
        long csize = cs[0] * cs[1] * cs[2];
        if (S->face_type[fc] == ORC_D) {
            memset(gc, 0, csize * sizeof(double));
            continue;
        }
        view_t vi = face_view(F->face_shape[fc]), vo = face_view(cs);
        restrict_view(S->restriction, S->g[l][fc], &vi, gc, &vo);
        long offx = 0, offy = 0, offz = 0, ii = 0, jj = 0, kk = 0, iii = 0, jjj = 0, kkk = 0;
        switch (fc) {
            case EAST: offx = F->shape[0] / 2; ii = -1; iii = -2; break;
            case WEST: ii = 1; iii = 2; break;
            case NORTH: offy = F->shape[1] / 2; jj = -1; jjj = -2; break;
            case SOUTH: jj = 1; jjj = 2; break;
            case TOP: offz = F->shape[2] / 2; kk = -1; kkk = -2; break;
            default: kk = 1; kkk = 2; break;
        }
        double c1 = -3.0 / 2.0, c2 = 2.0, c3 = -0.5;
        if (fc == EAST || fc == NORTH || fc == TOP) {
            c3 = 0.5;
            c2 = -2.0;
            c1 = 3.0 / 2.0;
        }
        const double h = F->h;
        const double* u = S->u[l];
        for (long i = 0; i < cs[0]; i++)
            for (long j = 0; j < cs[1]; j++)
                for (long k = 0; k < cs[2]; k++) {
                    long a = 2 * (i + offx), b = 2 * (j + offy), c = 2 * (k + offz);
                    gc[FIDX(cs, i, j, k)] -= (c1 * u[IDX(F, a, b, c)] + c2 * u[IDX(F, a + ii, b + jj, c + kk)] +
                                              c3 * u[IDX(F, a + iii, b + jjj, c + kkk)]) / h;
                }
    }
}

/* TrilinearInterpolation::prolong(u_{l+1} -> r_l) (include/trilinearinterpolation.h:29-134):
 * inject, then x, y and z midpoint passes. */
void orc_prolong(orc_solver* S, int l) {
    orc_level* F = &S->lv[l];
    orc_level* C = &S->lv[l + 1];
    const double* in = S->u[l + 1];
    double* out = S->r[l];
    for (long i = 0; i < C->shape[0]; i++)
        for (long j = 0; j < C->shape[1]; j++)
            for (long k = 0; k < C->shape[2]; k++) out[IDX(F, 2 * i, 2 * j, 2 * k)] = in[IDX(C, i, j, k)];
    for (long i = 1; i < F->shape[0] - 1; i += 2)
        for (long j = 0; j < F->shape[1]; j += 2)
            for (long k = 0; k < F->shape[2]; k += 2)
                out[IDX(F, i, j, k)] = 0.5 * (out[IDX(F, i - 1, j, k)] + out[IDX(F, i + 1, j, k)]);
    for (long i = 0; i < F->shape[0]; i++)
        for (long j = 1; j < F->shape[1] - 1; j += 2)
            for (long k = 0; k < F->shape[2]; k += 2)
                out[IDX(F, i, j, k)] = 0.5 * (out[IDX(F, i, j - 1, k)] + out[IDX(F, i, j + 1, k)]);
    for (long i = 0; i < F->shape[0]; i++)
        for (long j = 0; j < F->shape[1]; j++)
            for (long k = 1; k < F->shape[2] - 1; k += 2)
                out[IDX(F, i, j, k)] = 0.5 * (out[IDX(F, i, j, k - 1)] + out[IDX(F, i, j, k + 1)]);
}

/* DeviceArray::add (include/devicearray.h:161-196): u += r over the shape. */
void orc_add(orc_solver* S, int l) {
    orc_level* L = &S->lv[l];
    for (long i = 0; i < L->shape[0]; i++)
        for (long j = 0; j < L->shape[1]; j++)
            for (long k = 0; k < L->shape[2]; k++) S->u[l][IDX(L, i, j, k)] += S->r[l][IDX(L, i, j, k)];
}

/* DeviceArray::infinity_norm (include/devicearray.h:198-240): max |a| over the shape. */
double orc_norm(orc_solver* S, int field, int l) {
    orc_level* L = &S->lv[l];
    const double* a = orc_field(S, field, l);
    double res = 0.0;
    for (long i = 0; i < L->shape[0]; i++)
        for (long j = 0; j < L->shape[1]; j++)
            for (long k = 0; k < L->shape[2]; k++) {
                double v = fabs(a[IDX(L, i, j, k)]);
                if (v > res) res = v;
            }
    return res;
}

static void coarse_correction_setup(orc_solver* S, int l) {
    orc_residual(S, l);
    orc_restrict(S, l);
    orc_zero_u(S, l + 1);
    orc_restrict_bc(S, l);
}

/* Vcycle<T> (include/vcycle.h:14-98). */
void orc_vcycle(orc_solver* S, int l, double omega, long nsmooth) {
    orc_relax(S, l, omega, nsmooth);
    if (l >= S->levels - 1) return;
    coarse_correction_setup(S, l);
    orc_vcycle(S, l + 1, omega, nsmooth);
    orc_prolong(S, l);
    orc_add(S, l);
    orc_relax(S, l, omega, nsmooth);
}

/* Fcycle<T> (include/fcycle.h:13-97). */
void orc_fcycle(orc_solver* S, int l, double omega, long nsmooth) {
    orc_relax(S, l, omega, nsmooth);
    coarse_correction_setup(S, l);
    if (l < S->levels - 2) orc_fcycle(S, l + 1, omega, nsmooth);
    orc_vcycle(S, l + 1, omega, nsmooth);
    orc_prolong(S, l);
    orc_add(S, l);
    if (l == 0) orc_vcycle(S, 0, omega, nsmooth);
}

double orc_default_omega(const orc_solver* S) {
    return S->relaxation == ORC_JACOBI ? 6.0 / 7.0 : 8.0 / 9.0; /* jacobi.h:28-31, gaussseidel.h:96-99 */
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* PoissonSolver::solve (include/libpoisson.h:237-357) without the prints.
 * cycle: 0 relaxation (the reference's loop body does no smoothing, :304-308),
 * 1 V-cycle, 2 F-cycle.  history[iter] receives each iteration's relative residual
 * (up to hist_len entries).  Returns the number of entries written. */
long orc_solve(orc_solver* S, int cycle, long nsmooth, double omega, long maxiter, long miniter, double tol,
               double maxtime, double* rel_res_out, double* iters_out, double* time_out, double* history,
               long hist_len) {
    double wtime = now_s();
    if (omega < 0) omega = orc_default_omega(S);
    double fnorm = orc_norm(S, ORC_F, 0);
    orc_residual(S, 0);
    double rnorm = orc_norm(S, ORC_R, 0);
    double rel_res = rnorm / fnorm;
    long iter, nh = 0;
    for (iter = 0; iter < maxiter; iter++) {
        if (cycle == 1) orc_vcycle(S, 0, omega, nsmooth);
        else if (cycle == 2) orc_fcycle(S, 0, omega, nsmooth);
        orc_residual(S, 0);
        double norm = orc_norm(S, ORC_R, 0);
        norm /= fnorm;
        if (history && nh < hist_len) history[nh++] = norm;
        if (iter >= miniter) {
            if (norm > 2.0 * rel_res) {
                rel_res = norm;
                break;
            } else if (fabs(norm - rel_res) < tol) {
                rel_res = norm;
                break;
            }
            if ((now_s() - wtime) > maxtime) break;
        }
        rel_res = norm;
    }
    *rel_res_out = rel_res;
    *iters_out = (double)iter;
    *time_out = now_s() - wtime;
    return nh;
}

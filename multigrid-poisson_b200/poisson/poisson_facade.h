// poisson_facade.h -- header-only C++ facade of the reference's public solver API over the
// C ABI of libmgp.so (include/mgp.h).
//
// Rebuilds, with the same names, members and behaviour, the host-side surface of
// eljens/multigrid-poisson that user code touches:
//   Poisson::Settings (include/settings.h:14-39), DomainSettings/Grid (src/domainsettings.cpp,
//   src/grid.cpp), parser (src/parser.cpp:3-50), Halo (include/halo.h), Array<T> and
//   DeviceArray<T> with halo-aware idx() (include/array.h:20-141, include/devicearray.h),
//   BoundaryCondition / Boundary<T> / Dirichlet<T> / Neumann<T> (include/boundary.h,
//   dirichlet.h, neumann.h), the plug-in tags Injection, FullWeighting,
//   TrilinearInterpolation, Jacobi, GaussSeidel, and PoissonSolver<T,R,P,S>
//   (include/libpoisson.h:28-67).
// Host arrays keep the reference's exact layout, so `get_rhs(0).at[f.idx(i,j,k)] = ...` and
// `get_top_bc(0).arr.at[...]` work unchanged; the level hierarchy itself lives on the GPU
// inside libmgp.so and every computation runs there.
//
// Link with -lmgp (multigrid-poisson_b200/mgp/libmgp.so).  Problem functions
// Poisson::ufun/ffun/dudxfun/dudyfun/dudzfun are link-time plug-ins, as in the reference
// (include/problem_definition.h).
#ifndef MGP_POISSON_FACADE_H
#define MGP_POISSON_FACADE_H

#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mgp.h"

namespace Poisson {

using double_t = double;
using float_t = float;
using uint_t = long int;
using int_t = long int;

#ifndef MIN
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#endif

// ---- errors -------------------------------------------------------------------------
inline void mgp_throw(int status) {
    if (status == MGP_OK) return;
    std::string msg = mgp_last_error();
    if (status == MGP_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(std::string(mgp_status_string(status)) + ": " + msg);
}

// ---- Settings (include/settings.h:14-39) ------------------------------------------------
class Settings {
   public:
    uint_t levels = 1;
    uint_t dims[3] = {3, 3, 3};
    uint_t maxiter = 100;
    uint_t miniter = 1;
    double_t tolerance = 1e-6;
    int_t host = -1;  // the reference's omp_get_initial_device(); unused by the engine
    int_t dev = 0;
    double_t lengthx = 3.1415;
    double_t h = 0.33;
#ifndef PROBLEM2
    double_t origin[3] = {-0.4, 0.21, 1.23};
#else
    double_t origin[3] = {-1, -1, -1};
#endif
    bool print_result = false;
    bool write_final_stats = false;
    std::string stats_file = "";
    Settings() {}
    Settings(const Settings&) = default;
    Settings& operator=(const Settings&) = default;
};

inline std::ostream& operator<<(std::ostream& os, const Settings& s) {
    os << "Settings:" << std::endl;
    os << "\tDomain size: (" << s.dims[0] << "," << s.dims[1] << "," << s.dims[2] << ")" << std::endl;
    os << "\tMax iterations: " << s.maxiter << std::endl;
    os << "\tTolerance " << s.tolerance << std::endl;
    os << "\tHost id: " << s.host << std::endl;
    os << "\tDevice id: " << s.host << std::endl;
    os << "\tSave result: " << s.print_result << std::endl;
    return os;
}

// DomainSettings(settings, l) (src/domainsettings.cpp:12-29)
class DomainSettings : public Settings {
   public:
    DomainSettings() : Settings() {}
    DomainSettings(const Settings& s, const uint_t l) : Settings(s) {
        if (l > 0) {
            const uint_t o[3] = {dims[0], dims[1], dims[2]};
            for (int k = 0; k < 3; k++) dims[k] = (dims[k] >> l) + 1;
            h *= (double_t)(1L << l);
            if ((((dims[0] - 1) << l) + 1 != o[0]) || (((dims[1] - 1) << l) + 1 != o[1]) ||
                (((dims[2] - 1) << l) + 1 != o[2]))
                throw std::invalid_argument("Invalid grid of size: (" + std::to_string(dims[0]) + "," +
                                            std::to_string(dims[1]) + "," + std::to_string(dims[2]) + ")");
        }
    }
};

inline std::ostream& operator<<(std::ostream& os, const DomainSettings& s) {
    os << "DomainSettings:" << std::endl;
    os << "\tDomain size: (" << s.dims[0] << "," << s.dims[1] << "," << s.dims[2] << ")" << std::endl;
    os << "\tGridSpacing: " << s.h << std::endl;
    return os;
}

// Grid (src/grid.cpp:6-13): one DomainSettings per level, printed as built.
class Grid {
   public:
    const uint_t levels;
    std::vector<DomainSettings> domainsettings;
    Grid(const Settings& s, const uint_t _levels) : levels(_levels) {
        for (uint_t l = 0; l < _levels; l++) {
            domainsettings.push_back(DomainSettings(s, l));
            std::cout << domainsettings[l];
        }
    }
};

// parser (src/parser.cpp:3-50): -x -y -z -tol/-tolerance -maxiter -l/-levels -s/-save
// -length -stats; h = lengthx/(nx-1).
inline Settings parser(int argc, char* argv[]) {
    Settings set;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> std::string {
            if (i + 1 >= argc) throw std::invalid_argument("missing value after " + a);
            return std::string(argv[++i]);
        };
        if (a == "-x") set.dims[0] = std::stoi(next());
        else if (a == "-y") set.dims[1] = std::stoi(next());
        else if (a == "-z") set.dims[2] = std::stoi(next());
        else if (a == "-tolerance" || a == "-tol") set.tolerance = std::stod(next());
        else if (a == "-maxiter") set.maxiter = std::stoi(next());
        else if (a == "-levels" || a == "-l") set.levels = std::stoi(next());
        else if (a == "-save" || a == "-s") set.print_result = true;
        else if (a == "-length") set.lengthx = std::stod(next());
        else if (a == "-stats") {
            set.stats_file = next();
            set.write_final_stats = true;
        } else std::cerr << "Unknown input " << a << std::endl;
    }
    set.h = set.lengthx / ((double_t)set.dims[0] - 1.0);
    return set;
}

// ---- Halo / Array / DeviceArray --------------------------------------------------------
class Halo {
   public:
    uint_t east, west, north, south, top, bottom;
    Halo() : east(0), west(0), north(0), south(0), top(0), bottom(0) {}
    Halo(uint_t e, uint_t w, uint_t n, uint_t s, uint_t t, uint_t b)
        : east(e), west(w), north(n), south(s), top(t), bottom(b) {}
};

inline constexpr uint_t idx(const uint_t i, const uint_t j, const uint_t k, const Halo& h, const uint_t (&s)[3]) {
    return (i + h.west) * s[0] + (j + h.south) * s[1] + (k + h.bottom) * s[2];
}
inline constexpr uint_t idx_halo(const uint_t i, const uint_t j, const uint_t k, const uint_t (&s)[3]) {
    return i * s[0] + j * s[1] + k * s[2];
}

template <class T>
class Array {
   public:
    T* at = nullptr;
    const uint_t ndims = 3;
    const uint_t size;
    const uint_t shape[3];
    const uint_t stride[3];
    const Halo halo;

    Array(uint_t i, uint_t j, uint_t k) : size(i * j * k), shape{i, j, k}, stride{j * k, k, 1}, halo() { alloc(); }
    Array(uint_t i, uint_t j, uint_t k, const Halo& h)
        : size((i + h.east + h.west) * (j + h.north + h.south) * (k + h.top + h.bottom)),
          shape{i, j, k},
          stride{(j + h.north + h.south) * (k + h.top + h.bottom), (k + h.top + h.bottom), 1},
          halo(h) {
        alloc();
    }
    Array(const Array&) = delete;
    Array& operator=(const Array&) = delete;
    virtual ~Array() { free_host(); }

    constexpr uint_t idx(const uint_t i, const uint_t j, const uint_t k) const {
        return Poisson::idx(i, j, k, halo, stride);
    }
    constexpr uint_t idx_halo(const uint_t i, const uint_t j, const uint_t k) const {
        return Poisson::idx_halo(i, j, k, stride);
    }

    void init_zero() {
        for (uint_t n = 0; n < size; n++) at[n] = 0.0;
    }
    void add(const Array<T>& a) {
        if (a.size != size) std::cerr << "Array size does not match in Array<T>.add()" << std::endl;
        for (uint_t i = 0; i < shape[0]; i++)
            for (uint_t j = 0; j < shape[1]; j++)
                for (uint_t k = 0; k < shape[2]; k++) at[idx(i, j, k)] += a.at[a.idx(i, j, k)];
    }
    T infinity_norm() const {
        T res = 0.0;
        for (uint_t i = 0; i < shape[0]; i++)
            for (uint_t j = 0; j < shape[1]; j++)
                for (uint_t k = 0; k < shape[2]; k++) res = std::max(res, (T)std::abs(at[idx(i, j, k)]));
        return res;
    }

    // Legacy VTK STRUCTURED_POINTS, binary big-endian (include/array.h:148-203).  The
    // scalar type tag and byte swap follow T (the reference always writes "double").
    void print(const Settings& settings, const char* fname) const { write_vtk(settings, fname, false); }
    void print_halo(const Settings& settings, const char* fname) const { write_vtk(settings, fname, true); }

   protected:
    bool pinned_ = false;
    void alloc() {
        void* p = nullptr;
        if (mgp_host_alloc(&p, (size_t)size * sizeof(T) + 1) == MGP_OK) {
            pinned_ = true;
            at = (T*)p;
        } else {
            at = new (std::nothrow) T[size];
            if (!at) std::cerr << "Memory allocation failed in Array" << std::endl;
        }
        if (at) std::memset(at, 0, (size_t)size * sizeof(T));
    }
    void free_host() {
        if (!at) return;
        if (pinned_) mgp_host_free(at);
        else delete[] at;
        at = nullptr;
    }
    void write_vtk(const Settings& settings, const char* fname, bool with_halo) const {
        FILE* fp = fopen(fname, "w");
        if (!fp) {
            perror("No output! fopen()");
            return;
        }
        const uint_t nx = with_halo ? shape[0] + halo.east + halo.west : shape[0];
        const uint_t ny = with_halo ? shape[1] + halo.north + halo.south : shape[1];
        const uint_t nz = with_halo ? shape[2] + halo.top + halo.bottom : shape[2];
        const uint_t items = nx * ny * nz;
        if (with_halo)
            std::cout << "Printing file " << fname << " with shape (" << nx << "," << ny << "," << nz << ")"
                      << std::endl;
        fprintf(fp, "# vtk DataFile Version 3.0\n");
        fprintf(fp, "saved from function print_vtk.\n");
        fprintf(fp, "BINARY\n");
        fprintf(fp, "DATASET STRUCTURED_POINTS\n");
        fprintf(fp, "DIMENSIONS %d %d %d\n", (int)nx, (int)ny, (int)nz);
        const double ox = with_halo ? settings.origin[0] - (double)halo.west * settings.h : settings.origin[0];
        const double oy = with_halo ? settings.origin[1] - (double)halo.south * settings.h : settings.origin[1];
        const double oz = with_halo ? settings.origin[2] - (double)halo.bottom * settings.h : settings.origin[2];
        fprintf(fp, "ORIGIN %f %f %f\n", ox, oy, oz);
        fprintf(fp, "SPACING %f %f %f\n", settings.h, settings.h, settings.h);
        fprintf(fp, "POINT_DATA %" PRIu64 "\n", (uint64_t)items);
        fprintf(fp, "SCALARS %s %s 1\n", "gray", sizeof(T) == 8 ? "double" : "float");
        fprintf(fp, "LOOKUP_TABLE default\n");
        uint_t written = 0;
        for (uint_t k = 0; k < nz; ++k)
            for (uint_t j = 0; j < ny; ++j)
                for (uint_t i = 0; i < nx; ++i) {
                    const T v = with_halo ? at[idx_halo(i, j, k)] : at[idx(i, j, k)];
                    unsigned char b[sizeof(T)];
                    std::memcpy(b, &v, sizeof(T));
                    const uint32_t one = 1;
                    if (*(const unsigned char*)&one == 1)
                        for (size_t q = 0; q < sizeof(T) / 2; q++) std::swap(b[q], b[sizeof(T) - 1 - q]);
                    written += fwrite(b, sizeof(T), 1, fp);
                }
        if (written != items) std::cerr << "Failed to print file " << fname << std::endl;
        fclose(fp);
    }
};

// Host side of a device array.  Device storage belongs to the solver that owns the array
// (libmgp.so keeps every level on the GPU); devptr stays null on the host facade.
template <class T>
class DeviceArray : public Array<T> {
   public:
    uint_t device;
    T* devptr = nullptr;
    DeviceArray(uint_t dev, uint_t i, uint_t j, uint_t k) : Array<T>(i, j, k), device(dev) {}
    DeviceArray(const Settings& s, const Halo& h) : Array<T>(s.dims[0], s.dims[1], s.dims[2], h), device(s.dev) {}
};

// ---- boundaries -------------------------------------------------------------------------
typedef enum { NORTH, SOUTH, EAST, WEST, TOP, BOTTOM } Location_t;
typedef enum { DIRICHLET, NEUMANN } Boundary_t;

typedef struct BoundaryCondition {
    Boundary_t north;
    Boundary_t south;
    Boundary_t east;
    Boundary_t west;
    Boundary_t top;
    Boundary_t bottom;
} BoundaryCondition;

typedef double_t (*funptr)(double_t x, double_t y, double_t z);
double_t ufun(double_t x, double_t y, double_t z);
double_t ffun(double_t x, double_t y, double_t z);
double_t dudxfun(double_t x, double_t y, double_t z);
double_t dudyfun(double_t x, double_t y, double_t z);
double_t dudzfun(double_t x, double_t y, double_t z);

template <class T>
class Boundary {
   public:
    Location_t location;
    DeviceArray<T> arr;
    Boundary(int_t device, Location_t loc, uint_t i, uint_t j, uint_t k) : location(loc), arr(device, i, j, k) {}
    virtual ~Boundary() {}
    virtual bool is_neumann() const = 0;
    virtual void init(funptr u, funptr dx, funptr dy, funptr dz, const Settings& s) = 0;
    void init_zero() { arr.init_zero(); }
    // Boundary::init_by_fun (include/boundary.h:81-111)
    void init_by_fun(funptr fun, const Settings& s) {
        const double_t x0 = s.origin[0], y0 = s.origin[1], z0 = s.origin[2], h = s.h;
        double_t offx = 0, offy = 0, offz = 0;
        if (location == TOP) offz = s.dims[2] - 1;
        if (location == NORTH) offy = s.dims[1] - 1;
        if (location == EAST) offx = s.dims[0] - 1;
        for (int_t i = 0; i < arr.shape[0]; i++)
            for (int_t j = 0; j < arr.shape[1]; j++)
                for (int_t k = 0; k < arr.shape[2]; k++)
                    arr.at[arr.idx(i, j, k)] = fun(x0 + (((double_t)i) + offx) * h, y0 + (((double_t)j) + offy) * h,
                                                   z0 + (((double_t)k) + offz) * h);
    }
};

template <class T>
class Dirichlet : public Boundary<T> {
   public:
    Dirichlet(int_t d, Location_t l, uint_t i, uint_t j, uint_t k) : Boundary<T>(d, l, i, j, k) {}
    bool is_neumann() const override { return false; }
    void init(funptr u, funptr, funptr, funptr, const Settings& s) override { this->init_by_fun(u, s); }
};

template <class T>
class Neumann : public Boundary<T> {
   public:
    Neumann(int_t d, Location_t l, uint_t i, uint_t j, uint_t k) : Boundary<T>(d, l, i, j, k) {}
    bool is_neumann() const override { return true; }
    void init(funptr, funptr dx, funptr dy, funptr dz, const Settings& s) override {
        // neumann.h:63-79: east/west take du/dx, north/south du/dy, top/bottom du/dz
        if (this->location == EAST || this->location == WEST) this->init_by_fun(dx, s);
        else if (this->location == NORTH || this->location == SOUTH) this->init_by_fun(dy, s);
        else this->init_by_fun(dz, s);
    }
};

// ---- operator plug-ins: tags mapped to the engine's kernels -----------------------------
template <class T>
class Restriction {};
template <class T>
class Injection : public Restriction<T> {
   public:
    static constexpr int32_t mgp_kind = MGP_INJECTION;
};
template <class T>
class FullWeighting : public Restriction<T> {
   public:
    static constexpr int32_t mgp_kind = MGP_FULLWEIGHTING;
};
template <class T>
class Prolongation {};
template <class T>
class TrilinearInterpolation : public Prolongation<T> {
   public:
    static constexpr int32_t mgp_kind = MGP_TRILINEAR;
};
template <class T>
class Relaxation {};
template <class T>
class Jacobi : public Relaxation<T> {
   public:
    static constexpr int32_t mgp_kind = MGP_JACOBI;
    constexpr T default_omega() { return 6.0 / 7.0; }
    constexpr bool requires_duplicate_solution() { return true; }
    constexpr int smoothing_multiplier() { return 1; }
};
template <class T>
class GaussSeidel : public Relaxation<T> {
   public:
    static constexpr int32_t mgp_kind = MGP_GAUSSSEIDEL;
    constexpr T default_omega() { return 8.0 / 9.0; }
    constexpr bool requires_duplicate_solution() { return false; }
    constexpr int smoothing_multiplier() { return 2; }
};

template <class T>
struct mgp_dtype_of;
template <>
struct mgp_dtype_of<double> {
    static constexpr int32_t value = MGP_F64;
};
template <>
struct mgp_dtype_of<float> {
    static constexpr int32_t value = MGP_F32;
};

// ---- PoissonSolver (include/libpoisson.h:28-67) -----------------------------------------
template <class T, template <class> class R, template <class> class P, template <class> class S>
class PoissonSolver {
   public:
    PoissonSolver(int_t dev_shape[3], Settings& s, BoundaryCondition& bc) : settings(s), BC(bc), grid(s, s.levels) {
        check_shape(dev_shape);
        alloc();
    }
    PoissonSolver(Settings& s, BoundaryCondition& bc) : settings(s), BC(bc), grid(s, s.levels) { alloc(); }
    PoissonSolver(int_t dev_shape[3], Settings& s)
        : settings(s), BC({NEUMANN, NEUMANN, NEUMANN, NEUMANN, DIRICHLET, DIRICHLET}), grid(s, s.levels) {
        check_shape(dev_shape);
        alloc();
    }
    PoissonSolver(const PoissonSolver&) = delete;
    PoissonSolver& operator=(const PoissonSolver&) = delete;
    ~PoissonSolver() {
        for (auto* b : faces) delete b;
        delete u;
        delete uprev;
        delete f;
        delete r;
        if (handle) mgp_destroy(handle);
    }

    // PoissonSolver::init (include/libpoisson.h:158-171): the problem plug-ins sampled on
    // the host at level 0; coarse levels stay zero on the device.
    void init() {
        for (auto* b : faces) b->init(&ufun, &dudxfun, &dudyfun, &dudzfun, settings);
        const T x0 = settings.origin[0], y0 = settings.origin[1], z0 = settings.origin[2];
        const T h = settings.h;
        for (int_t i = 0; i < f->shape[0]; i++)
            for (int_t j = 0; j < f->shape[1]; j++)
                for (int_t k = 0; k < f->shape[2]; k++)
                    f->at[f->idx(i, j, k)] = ffun(x0 + ((T)i) * h, y0 + ((T)j) * h, z0 + ((T)k) * h);
        u->init_zero();
        uprev->init_zero();
        r->init_zero();
    }
    void init_zero() {
        for (auto* b : faces) b->init_zero();
        f->init_zero();
        u->init_zero();
        uprev->init_zero();
        r->init_zero();
    }
    // Domain::to_device (include/domain.h:245-263)
    void to_device() {
        mgp_throw(mgp_upload_field(handle, MGP_FIELD_U, 0, u->at, u->size));
        if (duplicate()) mgp_throw(mgp_upload_field(handle, MGP_FIELD_UPREV, 0, uprev->at, uprev->size));
        mgp_throw(mgp_upload_field(handle, MGP_FIELD_F, 0, f->at, f->size));
        mgp_throw(mgp_upload_field(handle, MGP_FIELD_R, 0, r->at, r->size));
        for (int fc = 0; fc < 6; fc++)
            mgp_throw(mgp_upload_face(handle, fc, 0, faces[fc]->arr.at, faces[fc]->arr.size));
        mgp_throw(mgp_write_bc(handle, 0));
    }
    // Domain::to_host (include/domain.h:265-272)
    void to_host() {
        mgp_throw(mgp_download_field(handle, MGP_FIELD_R, 0, r->at, r->size));
        mgp_throw(mgp_download_field(handle, MGP_FIELD_U, 0, u->at, u->size));
        if (duplicate()) mgp_throw(mgp_download_field(handle, MGP_FIELD_UPREV, 0, uprev->at, uprev->size));
    }
    void verbose(bool onoff) { is_verbose = onoff; }
    void solve(const std::string solver = "Vcycle", const int_t nsmooth = 10, T omega = -1.0, std::string ofile = "",
               double maxtime = 20 * 60) {
        int cyc;
        if (solver == "vcycle" || solver == "Vcycle") cyc = MGP_CYCLE_V;
        else if (solver == "fcycle" || solver == "Fcycle") cyc = MGP_CYCLE_F;
        else if (solver == "relaxation" || solver == "Relaxation") cyc = MGP_CYCLE_RELAXATION;
        else
            throw std::invalid_argument("solver must be \"Relaxation\", \"Vcycle\" of \"Fcycle\" but was \"" + solver +
                                        "\"");
        if (omega < 0) omega = relaxation.default_omega();
        mgp_stats st{};
        const uint32_t flags = MGP_SOLVE_PRINT_CYCLE_TIME | (is_verbose ? MGP_SOLVE_VERBOSE : 0u);
        mgp_throw(mgp_solve(handle, cyc, nsmooth, (double)omega, ofile.c_str(), maxtime, flags, &st));
        rel_res = st.rel_res;
        wtime = st.seconds;
        iter = (uint_t)st.iterations;
    }
    void save(uint_t gpuid, std::string file_name = "u.vtk") {
        u->print(grid.domainsettings[0], file_name.c_str());
        std::cout << "Saved " << file_name << std::endl;
    }
    void save_all(uint_t gpuid, std::string ufile = "u.vtk", std::string ffile = "f.vtk", std::string rfile = "r.vtk") {
        save_all(ufile, ffile, rfile);
    }
    void save_all(std::string ufile = "u.vtk", std::string ffile = "f.vtk", std::string rfile = "r.vtk") {
        u->print(grid.domainsettings[0], ufile.c_str());
        std::cout << "Saved " << ufile << std::endl;
        f->print(grid.domainsettings[0], ffile.c_str());
        std::cout << "Saved " << ffile << std::endl;
        r->print(grid.domainsettings[0], rfile.c_str());
        std::cout << "Saved " << rfile << std::endl;
    }
    T relative_residual() { return rel_res; }
    T solve_time() { return wtime; }
    T solve_iterations() { return iter; }
    DeviceArray<T>& get_rhs(uint_t gpuid) { return *f; }
    const DeviceArray<T>& get_solution(uint_t gpuid) { return *u; }
    const DeviceArray<T>& get_residual(uint_t gpuid) { return *r; }
    Boundary<T>& get_top_bc(uint_t gpuid) { return *faces[TOP]; }
    Boundary<T>& get_bottom_bc(uint_t gpuid) { return *faces[BOTTOM]; }
    // The engine's handle, for callers that drive the C ABI directly.
    mgp_solver* engine() { return handle; }

   private:
    Settings settings;
    BoundaryCondition BC;
    Grid grid;
    R<T> restriction_type;
    P<T> prolongation;
    S<T> relaxation;
    bool is_verbose = false;
    uint_t iter = 0;
    double_t rel_res = 0.0;
    double_t wtime = 0.0;
    mgp_solver* handle = nullptr;
    DeviceArray<T>*u = nullptr, *uprev = nullptr, *f = nullptr, *r = nullptr;
    Boundary<T>* faces[6] = {};

    bool duplicate() { return relaxation.requires_duplicate_solution(); }

    static void check_shape(int_t ds[3]) {
        if (ds[0] * ds[1] * ds[2] != 1)
            throw std::invalid_argument(
                "this engine solves one domain per GPU: dev_shape must be {1,1,1} (run one solver per GPU)");
    }

    void alloc() {
        mgp_desc d{};
        for (int k = 0; k < 3; k++) {
            d.dims[k] = settings.dims[k];
            d.origin[k] = settings.origin[k];
        }
        d.levels = settings.levels;
        d.maxiter = settings.maxiter;
        d.miniter = settings.miniter;
        d.tolerance = settings.tolerance;
        d.h = settings.h;
        const Boundary_t b[6] = {BC.north, BC.south, BC.east, BC.west, BC.top, BC.bottom};
        for (int k = 0; k < 6; k++) d.bc[k] = b[k] == NEUMANN ? MGP_NEUMANN : MGP_DIRICHLET;
        d.restriction = R<T>::mgp_kind;
        d.prolongation = P<T>::mgp_kind;
        d.relaxation = S<T>::mgp_kind;
        d.dtype = mgp_dtype_of<T>::value;
        d.device = (int32_t)settings.dev;
        mgp_throw(mgp_create(&d, &handle));
        mgp_level_info li{};
        mgp_throw(mgp_level_info_get(handle, 0, &li));
        const Halo halo(li.halo[0], li.halo[1], li.halo[2], li.halo[3], li.halo[4], li.halo[5]);
        u = new DeviceArray<T>(settings, halo);
        uprev = new DeviceArray<T>(settings, halo);
        f = new DeviceArray<T>(settings, halo);
        r = new DeviceArray<T>(settings, halo);
        const Location_t locs[6] = {NORTH, SOUTH, EAST, WEST, TOP, BOTTOM};
        for (int fc = 0; fc < 6; fc++) {
            const int64_t* fs = li.face_shape[fc];
            if (li.face_kind[fc] == MGP_NEUMANN) faces[fc] = new Neumann<T>(settings.dev, locs[fc], fs[0], fs[1], fs[2]);
            else faces[fc] = new Dirichlet<T>(settings.dev, locs[fc], fs[0], fs[1], fs[2]);
        }
    }
};

}  // namespace Poisson

// The reference's libpoisson.h exports these names to the global namespace
// (include/libpoisson.h:19-25); drivers rely on them.
using std::cout;
using std::endl;
using std::ios;
using std::ofstream;
using std::setw;
using std::string;
using Poisson::DIRICHLET;
using Poisson::NEUMANN;

#endif  // MGP_POISSON_FACADE_H

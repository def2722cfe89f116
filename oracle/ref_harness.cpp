// Reference harness -- TEST INFRASTRUCTURE ONLY, never part of the product path.
//
// Drives the reference's own Poisson::PoissonSolver<double,R,TrilinearInterpolation,S>
// (eljens/multigrid-poisson, header-only C++17 + OpenMP target regions) on the CPU and
// dumps its complete level hierarchy, so that
//   * the C restatement in oracle/mgp_oracle.c can be pinned bit-for-bit against the
//     reference itself, and
//   * the CUDA engine's parity tests have golden vectors generated by the reference.
//
// The reference sources are NOT copied: oracle/build_ref.sh compiles this file against the
// reference's include/ and src/ directories where they lie.  With no offload device the
// OpenMP target regions fall back to the host; the one-line omp_get_num_devices() shim
// below makes DeviceArray::device_allocator (include/devicearray.h:115-130) accept
// device 0, which libgomp then treats as the initial (host) device, so omp_target_alloc
// becomes a host allocation and "device" memory (devptr) is ordinary host memory.
//
// Input: a spec file of "key value..." lines (see parse_spec).  Output: raw little-endian
// double dumps of every level's u/uprev/f/r (full halo-padded arrays, the reference's own
// layout, include/array.h:70-77) and face arrays, a meta.txt describing the layout, and a
// stats.txt with %.17g numbers.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

// The harness reads the solver's level hierarchy (PoissonSolver::domains, private) and
// calls its operator objects directly; the reference's headers are otherwise unmodified.
#define private public
#define protected public
#include "libpoisson.h"
#undef private
#undef protected

extern "C" int omp_get_num_devices(void) { return 1; }

// ---------------------------------------------------------------------------------------
// Problem plug-ins.  The reference selects ufun/ffun/du*fun at link time
// (include/problem_definition.h:8-18, src/problem_definition.cpp); here one binary serves
// all problems through a run-time switch.
//   0  zero problem (u = f = g = 0)
//   1  reference PROBLEM1  sin(3x) sin(5.3y) sin(-7.8z)
//   2  reference PROBLEM2  x^3 y^2 z
//   3  reference PROBLEM3  cos(x z^2) sin(y^3)
//   10 sin(2 pi x) sin(2 pi y) sin(2 pi z), f = -12 pi^2 u (the 65^3 all-Dirichlet case)
static int g_problem = 0;
static const double kPi = 3.14159265358979323846;

namespace Poisson {
double_t ufun(double_t x, double_t y, double_t z) {
    switch (g_problem) {
        case 1: return sin(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return x * x * x * y * y * z;
        case 3: return cos(x * z * z) * sin(y * y * y);
        case 10: return sin(2.0 * kPi * x) * sin(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
double_t ffun(double_t x, double_t y, double_t z) {
    switch (g_problem) {
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
double_t dudxfun(double_t x, double_t y, double_t z) {
    switch (g_problem) {
        case 1: return 3.0 * cos(3.0 * x) * sin(5.3 * y) * sin(-7.8 * z);
        case 2: return 3.0 * x * x * y * y * z;
        case 3: return -z * z * sin(x * z * z) * sin(y * y * y);
        case 10: return 2.0 * kPi * cos(2.0 * kPi * x) * sin(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
double_t dudyfun(double_t x, double_t y, double_t z) {
    switch (g_problem) {
        case 1: return 5.3 * sin(3.0 * x) * cos(5.3 * y) * sin(-7.8 * z);
        case 2: return 2.0 * x * x * x * y * z;
        case 3: return 3.0 * cos(x * z * z) * y * y * cos(y * y * y);
        case 10: return 2.0 * kPi * sin(2.0 * kPi * x) * cos(2.0 * kPi * y) * sin(2.0 * kPi * z);
        default: return 0.0;
    }
}
double_t dudzfun(double_t x, double_t y, double_t z) {
    switch (g_problem) {
        case 1: return -7.8 * sin(3.0 * x) * sin(5.3 * y) * cos(-7.8 * z);
        case 2: return x * x * x * y * y;
        case 3: return -2 * x * z * sin(x * z * z) * sin(y * y * y);
        case 10: return 2.0 * kPi * sin(2.0 * kPi * x) * sin(2.0 * kPi * y) * cos(2.0 * kPi * z);
        default: return 0.0;
    }
}
}  // namespace Poisson

using Poisson::BoundaryCondition;
using Poisson::DeviceArray;
using Poisson::Domain;

// ---------------------------------------------------------------------------------------
struct Spec {
    long dims[3] = {17, 17, 17};
    long levels = 3;
    long maxiter = 10;
    long miniter = 1;
    double tolerance = 1e-6;
    double h = -1.0;  // <0: 1/(dims[0]-1)
    double origin[3] = {0.0, 0.0, 0.0};
    int bc[6] = {0, 0, 0, 0, 0, 0};  // north south east west top bottom; 0 D, 1 N
    std::string restriction = "inj";
    std::string relaxation = "gs";
    int problem = 0;  // -1: init_zero()
    std::string mode = "solve";
    std::string cycle = "Fcycle";
    long nsmooth = 2;
    double omega = -1.0;
    double maxtime = 1200.0;
    std::string load, out, ofile;
    std::vector<std::string> ops;
    long warm = 1, timed = 3;
    int verbose = 0;
};

static Spec parse_spec(const char* path) {
    Spec s;
    std::ifstream in(path);
    if (!in) throw std::runtime_error(std::string("cannot open spec ") + path);
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string key;
        if (!(ls >> key) || key[0] == '#') continue;
        if (key == "dims") ls >> s.dims[0] >> s.dims[1] >> s.dims[2];
        else if (key == "levels") ls >> s.levels;
        else if (key == "maxiter") ls >> s.maxiter;
        else if (key == "miniter") ls >> s.miniter;
        else if (key == "tolerance") ls >> s.tolerance;
        else if (key == "h") ls >> s.h;
        else if (key == "origin") ls >> s.origin[0] >> s.origin[1] >> s.origin[2];
        else if (key == "bc") {
            for (int f = 0; f < 6; f++) {
                std::string t;
                ls >> t;
                s.bc[f] = (t == "N" || t == "n" || t == "1") ? 1 : 0;
            }
        } else if (key == "restriction") ls >> s.restriction;
        else if (key == "relaxation") ls >> s.relaxation;
        else if (key == "problem") ls >> s.problem;
        else if (key == "mode") ls >> s.mode;
        else if (key == "cycle") ls >> s.cycle;
        else if (key == "nsmooth") ls >> s.nsmooth;
        else if (key == "omega") ls >> s.omega;
        else if (key == "maxtime") ls >> s.maxtime;
        else if (key == "load") ls >> s.load;
        else if (key == "out") ls >> s.out;
        else if (key == "ofile") ls >> s.ofile;
        else if (key == "warm") ls >> s.warm;
        else if (key == "timed") ls >> s.timed;
        else if (key == "verbose") ls >> s.verbose;
        else if (key == "ops") {
            std::string op;
            while (ls >> op) s.ops.push_back(op);
        } else throw std::runtime_error("unknown spec key " + key);
    }
    if (s.h < 0) s.h = 1.0 / (double)(s.dims[0] - 1);
    return s;
}

static const char* kFaceName[6] = {"north", "south", "east", "west", "top", "bottom"};

// ---------------------------------------------------------------------------------------
struct Runner {
    virtual ~Runner() {}
    virtual Poisson::Settings& settings() = 0;
    virtual Domain<double>& dom(long l) = 0;
    virtual void init(bool zero) = 0;
    virtual void to_device() = 0;
    virtual void to_host() = 0;
    virtual void solve(const std::string& cyc, long nsmooth, double omega, const std::string& ofile,
                       double maxtime) = 0;
    virtual double rel_res() = 0;
    virtual double iters() = 0;
    virtual double time() = 0;
    virtual void relax(long l, double omega, long nsmooth) = 0;
    virtual void restrict_r(long l) = 0;       // r_l -> f_{l+1}
    virtual void restrict_bc(long l) = 0;      // 6 boundary restrictions level l -> l+1
    virtual void prolong(long l) = 0;          // u_{l+1} -> r_l
    virtual void cycle(const std::string& c, long l, double omega, long nsmooth) = 0;
    virtual double default_omega() = 0;
    virtual bool duplicate() = 0;
    virtual void set_verbose(bool on) = 0;  // PoissonSolver::verbose (include/libpoisson.h:231-234)
};

template <template <class> class R, template <class> class S>
struct RunnerT : Runner {
    Poisson::PoissonSolver<double, R, Poisson::TrilinearInterpolation, S> solver;
    RunnerT(Poisson::Settings& st, BoundaryCondition& bc) : solver(st, bc) {}
    Poisson::Settings& settings() override { return solver.settings; }
    Domain<double>& dom(long l) override { return *solver.domains[0][l]; }
    void init(bool zero) override {
        if (zero) solver.init_zero();
        else solver.init();
    }
    void to_device() override { solver.to_device(); }
    void to_host() override { solver.to_host(); }
    void solve(const std::string& cyc, long nsmooth, double omega, const std::string& ofile,
               double maxtime) override {
        solver.solve(cyc, nsmooth, omega, ofile, maxtime);
    }
    void set_verbose(bool on) override { solver.verbose(on); }
    double rel_res() override { return solver.relative_residual(); }
    double iters() override { return solver.solve_iterations(); }
    double time() override { return solver.solve_time(); }
    void relax(long l, double omega, long nsmooth) override {
        // Through the base class, as the cycles call it (GaussSeidel hides relax()).
        static_cast<Poisson::Relaxation<double>&>(solver.relaxation).relax(solver.domains, omega, nsmooth, l, 1);
    }
    void restrict_r(long l) override {
        solver.restriction_type.restrict_to(*solver.domains[0][l]->r, *solver.domains[0][l + 1]->f);
    }
    void restrict_bc(long l) override {
        // Same six calls, same order, as include/vcycle.h:52-75.
        Domain<double>& fine = *solver.domains[0][l];
        Domain<double>& coarse = *solver.domains[0][l + 1];
        coarse.north->restrict_to(*fine.u, *fine.north, fine.settings, solver.restriction_type);
        coarse.south->restrict_to(*fine.u, *fine.south, fine.settings, solver.restriction_type);
        coarse.east->restrict_to(*fine.u, *fine.east, fine.settings, solver.restriction_type);
        coarse.west->restrict_to(*fine.u, *fine.west, fine.settings, solver.restriction_type);
        coarse.top->restrict_to(*fine.u, *fine.top, fine.settings, solver.restriction_type);
        coarse.bottom->restrict_to(*fine.u, *fine.bottom, fine.settings, solver.restriction_type);
    }
    void prolong(long l) override {
        solver.prolongation.prolong(*solver.domains[0][l + 1]->u, *solver.domains[0][l]->r);
    }
    void cycle(const std::string& c, long l, double omega, long nsmooth) override {
        if (c == "Vcycle")
            Poisson::Vcycle<double>(solver.domains, solver.restriction_type, solver.prolongation,
                                    solver.relaxation, omega, l, solver.settings.levels, 1, nsmooth);
        else
            Poisson::Fcycle<double>(solver.domains, solver.restriction_type, solver.prolongation,
                                    solver.relaxation, omega, l, solver.settings.levels, 1, nsmooth);
    }
    double default_omega() override { return solver.relaxation.default_omega(); }
    bool duplicate() override { return solver.relaxation.requires_duplicate_solution(); }
};

static Runner* make_runner(const Spec& s, Poisson::Settings& st, BoundaryCondition& bc) {
    bool fw = (s.restriction == "fw");
    bool jac = (s.relaxation == "jacobi");
    if (fw && jac) return new RunnerT<Poisson::FullWeighting, Poisson::Jacobi>(st, bc);
    if (fw) return new RunnerT<Poisson::FullWeighting, Poisson::GaussSeidel>(st, bc);
    if (jac) return new RunnerT<Poisson::Injection, Poisson::Jacobi>(st, bc);
    return new RunnerT<Poisson::Injection, Poisson::GaussSeidel>(st, bc);
}

// ---------------------------------------------------------------------------------------
static DeviceArray<double>* field(Domain<double>& d, const std::string& name) {
    if (name == "u") return d.u;
    if (name == "uprev") return d.uprev;
    if (name == "f") return d.f;
    if (name == "r") return d.r;
    throw std::runtime_error("unknown field " + name);
}

static Poisson::Boundary<double>* face(Domain<double>& d, int loc) {
    switch (loc) {
        case 0: return d.north;
        case 1: return d.south;
        case 2: return d.east;
        case 3: return d.west;
        case 4: return d.top;
        default: return d.bottom;
    }
}

static void write_raw(const std::string& path, const double* p, long n) {
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) throw std::runtime_error("cannot write " + path);
    if ((long)fwrite(p, sizeof(double), n, fp) != n) throw std::runtime_error("short write " + path);
    fclose(fp);
}

static bool read_raw(const std::string& path, double* p, long n) {
    FILE* fp = fopen(path.c_str(), "rb");
    if (!fp) return false;
    long got = (long)fread(p, sizeof(double), n, fp);
    fclose(fp);
    if (got != n) throw std::runtime_error("short read " + path);
    return true;
}

static void dump_meta(Runner& R, long levels, const std::string& dir) {
    std::ofstream m(dir + "/meta.txt");
    m.precision(17);
    for (long l = 0; l < levels; l++) {
        Domain<double>& d = R.dom(l);
        DeviceArray<double>& u = *d.u;
        m << "level " << l << " shape " << u.shape[0] << " " << u.shape[1] << " " << u.shape[2]
          << " halo " << u.halo.east << " " << u.halo.west << " " << u.halo.north << " " << u.halo.south
          << " " << u.halo.top << " " << u.halo.bottom << " stride " << u.stride[0] << " " << u.stride[1]
          << " " << u.stride[2] << " size " << u.size << " h " << d.settings.h << " faces";
        for (int f = 0; f < 6; f++) {
            Poisson::Boundary<double>* b = face(d, f);
            bool neu = dynamic_cast<Poisson::Neumann<double>*>(b) != nullptr;
            m << " " << (neu ? "N" : "D");
        }
        m << "\n";
    }
}

// Dump the "device" copies (devptr): with no offload device these are host memory and hold
// the solver's working state, whether or not to_host() was called.
static void dump_state(Runner& R, long levels, const std::string& dir) {
    dump_meta(R, levels, dir);
    for (long l = 0; l < levels; l++) {
        Domain<double>& d = R.dom(l);
        for (const char* fn : {"u", "uprev", "f", "r"}) {
            DeviceArray<double>* a = field(d, fn);
            write_raw(dir + "/L" + std::to_string(l) + "_" + fn + ".bin", a->devptr, a->size);
        }
        for (int f = 0; f < 6; f++) {
            DeviceArray<double>& a = face(d, f)->arr;
            write_raw(dir + "/L" + std::to_string(l) + "_" + kFaceName[f] + ".bin", a.devptr, a.size);
        }
    }
}

// Load whatever state files exist into the host copies (at); missing files keep the
// current contents.
static void load_host(Runner& R, long levels, const std::string& dir) {
    for (long l = 0; l < levels; l++) {
        Domain<double>& d = R.dom(l);
        for (const char* fn : {"u", "uprev", "f", "r"}) {
            DeviceArray<double>* a = field(d, fn);
            read_raw(dir + "/L" + std::to_string(l) + "_" + fn + ".bin", a->at, a->size);
        }
        for (int f = 0; f < 6; f++) {
            DeviceArray<double>& a = face(d, f)->arr;
            read_raw(dir + "/L" + std::to_string(l) + "_" + kFaceName[f] + ".bin", a.at, a.size);
        }
    }
}

// Copy every array's host copy to its device copy without writing boundary data into u
// (the raw half of Domain::to_device, include/domain.h:245-258).
static void raw_to_device(Runner& R, long levels) {
    for (long l = 0; l < levels; l++) {
        Domain<double>& d = R.dom(l);
        d.u->to_device();
        if (R.duplicate()) d.uprev->to_device();
        d.f->to_device();
        d.r->to_device();
        for (int f = 0; f < 6; f++) face(d, f)->arr.to_device();
    }
}

static void run_ops(Runner& R, const Spec& s, std::ostream& stats) {
    double omega = s.omega < 0 ? R.default_omega() : s.omega;
    double fnorm = 0.0;
    for (const std::string& opspec : s.ops) {
        std::string op = opspec;
        long l = 0;
        size_t c = opspec.find(':');
        if (c != std::string::npos) {
            op = opspec.substr(0, c);
            l = std::stol(opspec.substr(c + 1));
        }
        Domain<double>& d = R.dom(l);
        if (op == "relax") R.relax(l, omega, s.nsmooth);
        else if (op == "residual") Poisson::residual<double>(d);
        else if (op == "restrict") R.restrict_r(l);
        else if (op == "zero") d.u->init_zero();
        else if (op == "bcrestrict") R.restrict_bc(l);
        else if (op == "prolong") R.prolong(l);
        else if (op == "add") d.u->add(*d.r);
        else if (op == "writebc") {
            d.write_bc_to(*d.u);
            if (R.duplicate()) d.write_bc_to(*d.uprev);
        } else if (op == "vcycle") R.cycle("Vcycle", l, omega, s.nsmooth);
        else if (op == "fcycle") R.cycle("Fcycle", l, omega, s.nsmooth);
        else if (op == "fnorm") {
            fnorm = d.f->infinity_norm();
            stats << "fnorm " << fnorm << "\n";
        } else if (op == "unorm") stats << "unorm " << d.u->infinity_norm() << "\n";
        else if (op == "rnorm") {
            double rn = d.r->infinity_norm();
            stats << "rnorm " << rn << " rel " << (fnorm != 0.0 ? rn / fnorm : 0.0) << "\n";
        } else throw std::runtime_error("unknown op " + op);
    }
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: %s <spec-file>\n", argv[0]);
        return 2;
    }
    try {
        Spec s = parse_spec(argv[1]);
        Poisson::Settings st;
        st.dims[0] = s.dims[0];
        st.dims[1] = s.dims[1];
        st.dims[2] = s.dims[2];
        st.levels = s.levels;
        st.maxiter = s.maxiter;
        st.miniter = s.miniter;
        st.tolerance = s.tolerance;
        st.h = s.h;
        st.origin[0] = s.origin[0];
        st.origin[1] = s.origin[1];
        st.origin[2] = s.origin[2];
        BoundaryCondition bc;
        bc.north = s.bc[0] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        bc.south = s.bc[1] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        bc.east = s.bc[2] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        bc.west = s.bc[3] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        bc.top = s.bc[4] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        bc.bottom = s.bc[5] ? Poisson::NEUMANN : Poisson::DIRICHLET;
        g_problem = s.problem < 0 ? 0 : s.problem;

        // Grid's constructor prints every level to cout (src/grid.cpp:11); keep stdout for
        // the solver's own prints only when asked.
        std::streambuf* saved = std::cout.rdbuf();
        std::ofstream devnull("/dev/null");
        if (!s.verbose) std::cout.rdbuf(devnull.rdbuf());
        Runner* R = make_runner(s, st, bc);
        std::ostringstream stats;
        stats.precision(17);

        if (s.mode == "ops") {
            R->init(true);
            if (!s.load.empty()) load_host(*R, s.levels, s.load);
            raw_to_device(*R, s.levels);
            run_ops(*R, s, stats);
        } else if (s.mode == "solve") {
            R->init(s.problem < 0);
            if (!s.load.empty()) load_host(*R, 1, s.load);
            if (s.verbose) R->set_verbose(true);  // the solve's own prints (verbose 1 keeps stdout)
            R->to_device();
            R->solve(s.cycle, s.nsmooth, s.omega, s.ofile, s.maxtime);
            R->to_host();
            stats << "rel_res " << R->rel_res() << "\n";
            stats << "iters " << R->iters() << "\n";
            stats << "time " << R->time() << "\n";
        } else if (s.mode == "time") {
            // CPU baseline: the reference's own solve() timed by its own solve_time()
            // (include/libpoisson.h:238,356); a warm-up solve first.
            R->init(s.problem < 0);
            R->to_device();
            R->settings().maxiter = s.warm;
            if (s.warm > 0) R->solve(s.cycle, s.nsmooth, s.omega, "", s.maxtime);
            R->settings().maxiter = s.timed;
            R->solve(s.cycle, s.nsmooth, s.omega, "", s.maxtime);
            stats << "rel_res " << R->rel_res() << "\n";
            stats << "iters " << R->iters() << "\n";
            stats << "time " << R->time() << "\n";
            stats << "threads " << omp_get_max_threads() << "\n";
        } else {
            throw std::runtime_error("unknown mode " + s.mode);
        }
        std::cout.rdbuf(saved);
        if (!s.out.empty()) {
            if (s.mode != "time") dump_state(*R, s.levels, s.out);
            std::ofstream so(s.out + "/stats.txt");
            so << stats.str();
        }
        std::cout << stats.str();
        delete R;
    } catch (std::exception& e) {
        fprintf(stderr, "ref_harness error: %s\n", e.what());
        return 1;
    }
    return 0;
}

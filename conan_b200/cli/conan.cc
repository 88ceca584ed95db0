// conan -- host CLI with the reference's `ic`, `run`, `cic` and `fof` commands
// on the GPU.
//
// Drop-in for the reference binary's sub-commands (src/base/main.cc:95-119):
// the same option tables (src/ic/main.cc:15-65, src/run/main.cc:20-61,
// src/cic/main.cc:17-32), the same header/history merge (src/base/header.cc:
// 22-28, src/base/history.cc), the same file contracts: `ic` writes
// <id>.density.init.conan with records density [, potential] [,
// displacement]; `run` reads its potential record and writes
// <id>.pos.<k>.conan every 10 steps (or IFRIT .bin / ASCII .txt),
// src/run/nbody.hh:135-218; `cic` reads <id>.pos.<m>.conan and writes
// <id>.rho.<m>.conan (src/cic/main.cc:43-79); `fof` reads a snapshot and
// writes the text file <id>.fof.<t>.txt (src/fof/fof.cc:282-333). The
// numerics run in libconan_pm.so.
//
// Options that only this build has (precision, noise source, gradient,
// device, periodic gather) are marked local: they are parsed like the others
// but never written into file headers, so files keep the reference's keys.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "conan_pm.h"

namespace {

typedef std::runtime_error Fail;

// ----------------------------------------------------------- options ----

struct Option {
    enum { CHECK = 1, VALUED = 2, LOCAL = 4 };
    int flags;
    std::string short_name, long_name, value, description;
    bool valued() const { return flags & VALUED; }
};

struct Argv {
    std::vector<Option> opts;
    std::string command_line;

    std::string operator[](const std::string &name) const {
        for (auto &o : opts)
            if (o.long_name == name) return o.value;
        throw Fail("Trying to find option [" + name + "], but no such option exists.");
    }
    template <typename T> T get(const std::string &name) const {
        std::istringstream ss((*this)[name]);
        T v{};
        ss >> v;
        return v;
    }
    bool flag(const std::string &name) const { return get<bool>(name); }

    // Argv::parse (src/base/argv.cc:42-99): -s / --long, valued options take
    // the next argument, flags become "1".
    void parse(int argc, char **argv) {
        command_line = argv[0];
        for (int i = 1; i < argc; ++i) command_line += std::string(" ") + argv[i];
        int n = 1;
        while (n < argc) {
            std::string arg(argv[n]);
            if (arg.empty() || arg[0] != '-')
                throw Fail("Don't know how to handle [" + arg + "]");
            bool is_long = arg.size() > 1 && arg[1] == '-';
            std::string name = arg.substr(is_long ? 2 : 1);
            Option *o = nullptr;
            for (auto &x : opts)
                if ((is_long ? x.long_name : x.short_name) == name && !name.empty()) o = &x;
            if (!o) throw Fail("Got the argument [" + arg + "], but no such option exists.");
            if (o->valued()) {
                if (argc - n < 2) throw Fail("Got the last argument [" + arg + "], but no value given.");
                o->value = argv[n + 1];
                o->flags |= Option::CHECK;
                n += 2;
            } else {
                o->value = "1";
                o->flags |= Option::CHECK;
                n += 1;
            }
        }
    }

    void print(std::ostream &out) const {
        for (auto &o : opts) {
            std::ostringstream s;
            s << "        --" << o.long_name;
            if (!o.short_name.empty()) s << " | -" << o.short_name;
            if (o.valued()) s << " (default: " << o.value << ")";
            else s << " (flag)";
            s << " : " << o.description;
            out << s.str() << "\n";
        }
    }
};

// ------------------------------------------------------- file blocks ----

void write_block(std::ostream &f, const void *data, uint64_t nbytes) {
    f.write(reinterpret_cast<const char *>(&nbytes), sizeof nbytes);
    f.write(reinterpret_cast<const char *>(data), (std::streamsize)nbytes);
    f.write(reinterpret_cast<const char *>(&nbytes), sizeof nbytes);
}

void write_block_32(std::ostream &f, const void *data, uint32_t nbytes) {
    f.write(reinterpret_cast<const char *>(&nbytes), sizeof nbytes);
    f.write(reinterpret_cast<const char *>(data), nbytes);
    f.write(reinterpret_cast<const char *>(&nbytes), sizeof nbytes);
}

std::vector<char> read_block(std::istream &f) {
    uint64_t a = 0, b = 0;
    f.read(reinterpret_cast<char *>(&a), sizeof a);
    if (f.fail()) throw Fail("Could not read from file");
    std::vector<char> v(a);
    f.read(v.data(), (std::streamsize)a);
    f.read(reinterpret_cast<char *>(&b), sizeof b);
    if (f.fail() || a != b) throw Fail("The block seems to be corrupted");
    return v;
}

void skip_block(std::istream &f) {
    uint64_t a = 0, b = 0;
    f.read(reinterpret_cast<char *>(&a), sizeof a);
    if (f.fail()) throw Fail("Could not read from file");
    f.seekg((std::streamoff)a, std::ios::cur);
    f.read(reinterpret_cast<char *>(&b), sizeof b);
    if (f.fail() || a != b) throw Fail("The block seems to be corrupted");
}

std::string first_line(const std::string &s) { return s.substr(0, s.find('\n')); }

// key=value lines in std::map order (src/base/header.cc:30-74).
struct Header : std::map<std::string, std::string> {
    Header &operator<<(const Argv &C) {
        for (auto &o : C.opts)
            if (!(o.flags & Option::LOCAL)) (*this)[o.long_name] = o.value;
        return *this;
    }
    template <typename T> T get(const std::string &name) const {
        auto i = find(name);
        if (i == end()) throw Fail("variable [" + name + "] not found in config.");
        std::istringstream ss(i->second);
        T v{};
        ss >> v;
        return v;
    }
    void to_file(std::ostream &f) const {
        std::ostringstream s;
        for (auto &kv : *this) s << kv.first << "=" << first_line(kv.second) << "\n";
        std::string out = s.str();
        write_block(f, out.data(), out.size());
    }
    void from_file(std::istream &f) {
        clear();
        auto raw = read_block(f);
        std::string in(raw.begin(), raw.end());
        size_t pos = 0;
        while (pos < in.size()) {
            size_t p1 = in.find('=', pos), p2 = in.find('\n', pos);
            if (p1 == std::string::npos || p2 == std::string::npos) break;
            insert({in.substr(pos, p1 - pos), in.substr(p1 + 1, p2 - p1 - 1)});
            pos = p2 + 1;
        }
    }
};

// time:command lines (src/base/history.cc:20-75).
struct History : std::multimap<long long, std::string> {
    void update(const std::string &cmd) { insert({(long long)time(nullptr), cmd}); }
    void to_file(std::ostream &f) const {
        std::ostringstream s;
        for (auto &kv : *this) s << kv.first << ":" << first_line(kv.second) << "\n";
        std::string out = s.str();
        write_block(f, out.data(), out.size());
    }
    void from_file(std::istream &f) {
        auto raw = read_block(f);
        std::string in(raw.begin(), raw.end());
        size_t pos = 0;
        while (pos < in.size()) {
            size_t p1 = in.find(':', pos), p2 = in.find('\n', pos);
            if (p1 == std::string::npos || p2 == std::string::npos) break;
            insert({std::stoll(in.substr(pos, p1 - pos)), in.substr(p1 + 1, p2 - p1 - 1)});
            pos = p2 + 1;
        }
    }
};

// dtype names of src/base/mtypeid.cc:49-64 for R doubles per element.
std::string dtype_f8(int R) {
    if (R == 1) return "float64";
    return std::to_string(R) + "f8";
}

void save_record(std::ostream &f, const std::string &name, const std::string &dtype, const void *data,
                 size_t nbytes) {
    Header S;
    S["name"] = name;
    S["dtype"] = dtype;
    S.to_file(f);
    write_block(f, data, nbytes);
}

std::vector<double> load_record(std::istream &fi, const std::string &name) {
    auto pos = fi.tellg();
    while (fi.good()) {
        Header S;
        S.from_file(fi);
        if (S["name"] != name) {
            skip_block(fi);
        } else {
            auto raw = read_block(fi);
            std::vector<double> v(raw.size() / sizeof(double));
            std::memcpy(v.data(), raw.data(), v.size() * sizeof(double));
            fi.seekg(pos, std::ios::beg);
            return v;
        }
    }
    throw Fail("Couldn't find record " + name + " in file.");
}

template <typename... A> std::string fmt(A &&...a) {
    std::ostringstream ss;
    (ss << ... << a);
    return ss.str();
}

std::string date_string() {
    time_t t = time(nullptr);
    struct tm *T = gmtime(&t);
    std::ostringstream s;
    s << std::setfill('0') << std::setw(2) << T->tm_year - 100 << std::setw(2) << T->tm_mon + 1
      << std::setw(2) << T->tm_mday;
    return s.str();
}

void check(int rc) {
    if (rc != CONAN_OK) throw Fail(conan_last_error());
}

int precision_of(const std::string &s) {
    if (s == "fp32" || s == "float32") return CONAN_FP32;
    if (s == "fp64" || s == "float64") return CONAN_FP64;
    throw Fail("precision must be fp32 or fp64, got [" + s + "]");
}

// --------------------------------------------------------------- ic ----

void cmd_ic(int argc, char **argv) {
    std::string timed_seed = std::to_string((long long)time(nullptr));
    Argv C;
    C.opts = {
        {0, "h", "help", "false", "print help on the use of this program."},
        {Option::VALUED | Option::CHECK, "i", "id", date_string(), "identifier for filenames."},
        {Option::VALUED | Option::CHECK, "d", "dim", "3",
         "number of dimensions in which to run the code. Usually this should by 2 or 3."},
        {Option::VALUED | Option::CHECK, "b", "mbits", "8",
         "size of the mass-box, or binary power of the number of particles per dimension."},
        {Option::VALUED | Option::CHECK, "L", "size", "100", "physical size of the simulation in units of Mpc/h."},
        {Option::VALUED | Option::CHECK, "", "seed", timed_seed,
         "random seed used to generate the initial conditions."},
        {Option::VALUED | Option::CHECK, "", "Omega0", "0.32", "matter density."},
        {Option::VALUED | Option::CHECK, "", "H0", "69.0", "Hubble parameter."},
        {Option::VALUED | Option::CHECK, "n", "ns", "0.96", "the slope of the power spectrum."},
        {0, "", "smooth", "false", "whether to smooth the initial conditions with a Gaussian filter or not."},
        {0, "", "scale-free", "false", "this will enable a scale-free power-spectrum with power law index <ns>."},
        {Option::VALUED | Option::CHECK, "", "scale", "8.0", "scale at which to smooth in units of Mpc/h."},
        {Option::VALUED | Option::CHECK, "", "sigma", "0.83", "normalisation at given scale."},
        {0, "p", "potential", "false", "include the potential in the result."},
        {0, "z", "displacement", "false", "include the Zel'dovich displacement in the result."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "precision", "fp64",
         "GPU mesh arithmetic: fp64 or fp32."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "noise", "mt19937",
         "white-noise source: mt19937 (the reference's generator, drawn on the host) or philox (GPU)."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "device", "0", "CUDA device."},
    };
    C.parse(argc, argv);
    if (C.flag("help")) {
        std::cout << "Cosmic workset Conan (B200 build).\n\n";
        C.print(std::cout);
        exit(0);
    }
    Header H;
    H << C;
    H["N"] = fmt(1 << H.get<unsigned>("mbits"));
    History I;
    I.update(C.command_line);

    conan_ic_params p{};
    p.dim = H.get<int>("dim");
    p.mbits = H.get<int>("mbits");
    p.size = H.get<double>("size");
    p.seed = H.get<unsigned>("seed");
    p.ns = H.get<double>("ns");
    p.smooth = H.get<bool>("smooth");
    p.scale_free = H.get<bool>("scale-free");
    p.scale = H.get<double>("scale");
    p.sigma = H.get<double>("sigma");
    p.Omega0 = H.get<double>("Omega0");
    p.H0 = H.get<double>("H0");
    p.precision = precision_of(C["precision"]);
    p.device = C.get<int>("device");
    if (p.dim < 1 || p.dim > 3) throw Fail("only 2 and 3 dimensions supported.");
    size_t n = (size_t)1 << ((size_t)p.mbits * p.dim);

    std::vector<double> D(n), noise;
    const double *nz = nullptr;
    if (C["noise"] == "mt19937") {
        // Gaussian_white_noise(seed), src/base/misc.hh:179-188: libstdc++'s
        // std::mt19937 and std::normal_distribution<double>, in memory order.
        std::mt19937 rng((unsigned)p.seed);
        std::normal_distribution<double> normal;
        noise.resize(n);
        for (auto &x : noise) x = normal(rng);
        nz = noise.data();
    } else if (C["noise"] != "philox") {
        throw Fail("noise must be mt19937 or philox");
    }
    check(conan_ic_generate(&p, nz, D.data()));

    std::ofstream fo(C["id"] + ".density.init.conan", std::ios::binary);
    if (!fo) throw Fail("could not open output file");
    H.to_file(fo);
    I.to_file(fo);
    save_record(fo, "density", "float64", D.data(), D.size() * sizeof(double));
    if (C.flag("potential")) {
        check(conan_ic_potential(&p, D.data()));
        save_record(fo, "potential", "float64", D.data(), D.size() * sizeof(double));
    }
    if (C.flag("displacement")) {
        if (p.dim < 2) throw Fail("only 2 and 3 dimensions supported.");
        std::vector<double> psi(n * p.dim);
        check(conan_ic_displacement(&p, D.data(), psi.data()));
        save_record(fo, "displacement", dtype_f8(p.dim), psi.data(), psi.size() * sizeof(double));
    }
}

// -------------------------------------------------------------- run ----

enum Format { FMT_ASCII, FMT_IFRIT, FMT_CONAN };

// Snapshot writing overlaps the GPU: the callback copies the state to host
// memory and hands it to a writer thread, then the run continues while the
// file is written; the next snapshot (and the end of the run) waits for the
// previous writer. At most two snapshots are held in host memory.
struct Snapshot {
    unsigned index;
    double a, a_pos, a_mom;
    std::vector<double> X, P;
};

struct RunCtx {
    std::string id;
    int dim;
    unsigned N;
    double L;
    Format format;
    size_t np;
    std::thread writer;
    std::string writer_error;

    void join() {
        if (writer.joinable()) writer.join();
        if (!writer_error.empty()) throw Fail(writer_error);
    }
};

void write_snapshot(const RunCtx &c, const Snapshot &s) {
    const char *ext = c.format == FMT_ASCII ? ".txt" : c.format == FMT_IFRIT ? ".bin" : ".conan";
    std::string fn = fmt(c.id, ".pos.", s.index, ext);
    std::ofstream fo(fn, std::ios::binary);
    if (!fo) throw Fail("could not open " + fn);
    const std::vector<double> &X = s.X, &P = s.P;
    if (c.format == FMT_ASCII) {
        // X[i] " " P[i]/a with mVector's trailing-space printing.
        for (size_t j = 0; j < c.np; ++j) {
            for (int k = 0; k < c.dim; ++k) fo << X[j * c.dim + k] << " ";
            fo << " ";
            for (int k = 0; k < c.dim; ++k) fo << P[j * c.dim + k] / s.a << " ";
            fo << "\n";
        }
    } else if (c.format == FMT_IFRIT) {
        uint32_t N = (uint32_t)c.np;
        write_block_32(fo, &N, 4);
        float dims[6] = {0, 0, 0, (float)c.L, (float)c.L, (float)c.L};
        write_block_32(fo, dims, sizeof dims);
        std::vector<float> data(c.np);
        for (int which = 0; which < 2; ++which)
            for (int k = 0; k < 3; ++k) {
                const std::vector<double> &src = which ? P : X;
                for (size_t j = 0; j < c.np; ++j) data[j] = (float)src[j * 3 + k];
                write_block_32(fo, data.data(), (uint32_t)(data.size() * sizeof(float)));
            }
    } else {
        Header H;
        H["id"] = c.id;
        H["N"] = fmt(c.N);
        H["L"] = fmt(c.L);
        H["dim"] = fmt(c.dim);
        H["a-mom"] = fmt(s.a_mom);
        H["a-pos"] = fmt(s.a_pos);
        History I;
        I.update("ran nbody");
        H.to_file(fo);
        I.to_file(fo);
        std::string dt = c.dim == 1 ? "" : dtype_f8(c.dim);
        save_record(fo, "pos", dt, X.data(), X.size() * sizeof(double));
        save_record(fo, "mom", dt, P.data(), P.size() * sizeof(double));
    }
    if (!fo) throw Fail("could not write " + fn);
}

void save_snapshot(conan_pm *h, RunCtx &c, unsigned i, double a) {
    std::cout << "|";
    std::cout.flush();
    if (c.format == FMT_IFRIT && c.dim != 3) throw Fail("IFRIT files only support 3D");
    auto s = std::make_shared<Snapshot>();
    s->index = (i + 1) / 10;
    s->a = a;
    s->X.resize(c.np * c.dim);
    s->P.resize(c.np * c.dim);
    check(conan_pm_get_state(h, s->X.data(), s->P.data()));
    check(conan_pm_scale_factors(h, &s->a_pos, &s->a_mom));
    c.join();  // the previous snapshot's file is complete
    c.writer = std::thread([&c, s] {
        try {
            write_snapshot(c, *s);
        } catch (std::exception &e) {
            c.writer_error = e.what();
        }
    });
}

struct CbData {
    RunCtx *ctx;
    std::string error;
    unsigned done = 0;
};

int step_cb(conan_pm *h, unsigned step, double a, void *user) {
    CbData *d = static_cast<CbData *>(user);
    for (; d->done <= step; ++d->done) std::cout << ".";
    std::cout.flush();
    try {
        if ((step + 1) % 10 == 0) save_snapshot(h, *d->ctx, step, a);
    } catch (std::exception &e) {
        d->error = e.what();
        return 1;
    }
    return 0;
}

void cmd_run(int argc, char **argv) {
    Argv C;
    C.opts = {
        {0, "h", "help", "false", "print help on the use of this program."},
        {Option::VALUED | Option::CHECK, "i", "id", date_string(), "identifier for filenames."},
        {Option::VALUED | Option::CHECK, "H0", "H0", "68.5", "Hubble parameter."},
        {Option::VALUED | Option::CHECK, "m", "Omega_m", "1.0", "Omega-matter. The default universe is EdS."},
        {Option::VALUED | Option::CHECK, "L", "Omega_L", "0.0", "Omega-Lambda. The default universe is EdS."},
        {0, "c", "concordance", "false",
         "Override cosmological parameters to have concordance (Planck) model: H0 = 68.5, Omega_L = 0.69, "
         "Omega_m = 0.31"},
        {Option::VALUED | Option::CHECK, "f", "f", "2",
         "fractional force resolution. The default makes the force grid twice the size of the mass grid."},
        {Option::VALUED | Option::CHECK, "a0", "a0", "0.02", "start time."},
        {Option::VALUED | Option::CHECK, "da", "da", "0.02", "size of time step."},
        {Option::VALUED | Option::CHECK, "n", "n", "50", "number of iterations."},
        {0, "", "flip-flops", "false", "count number of flip-flops for each particle."},
        {0, "", "ifrit", "false", "give output in Ifrit readable format."},
        {0, "", "ascii", "false", "give output in ASCII (not recommended for 3D)."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "precision", "fp32",
         "GPU particle and mesh arithmetic: fp32 (lattice index + FP32 displacement) or fp64."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "gradient", "fd4",
         "force gradient: fd4 (the reference's 4-point difference) or spectral."},
        {0 | Option::LOCAL, "", "periodic-gather", "false",
         "interpolate forces with periodic floor indices instead of the reference's truncation."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "device", "0", "CUDA device."},
    };
    C.parse(argc, argv);
    if (C.flag("help")) {
        std::cout << "Cosmic workset Conan (B200 build).\n\n";
        C.print(std::cout);
        exit(0);
    }
    std::ifstream fi(C["id"] + ".density.init.conan", std::ios::binary);
    if (!fi) throw Fail("Could not read from file");
    Header H;
    H.from_file(fi);
    H << C;
    History I;
    I.from_file(fi);
    I.update(C.command_line);
    std::vector<double> phi = load_record(fi, "potential");
    fi.close();

    unsigned f = H.get<unsigned>("f"), N = H.get<unsigned>("N");
    double L = H.get<double>("size");
    double H0 = H.get<double>("H0"), Om = H.get<double>("Omega_m"), OL = H.get<double>("Omega_L");
    if (C.flag("concordance")) {
        H0 = 68.5;
        Om = 0.31;
        OL = 0.69;
    }
    double a0 = H.get<double>("a0"), da = H.get<double>("da");
    unsigned n = (unsigned)H.get<double>("n");
    Format format = FMT_CONAN;
    if (H.get<bool>("ifrit")) format = FMT_IFRIT;
    if (H.get<bool>("ascii")) format = FMT_ASCII;
    int dim = H.get<int>("dim");

    conan_pm_params p{};
    p.dim = dim;
    p.n_mass = (int)N;
    p.f = (int)f;
    p.size = L;
    p.H0 = H0;
    p.Omega_m = Om;
    p.Omega_L = OL;
    p.precision = precision_of(C["precision"]);
    if (C["gradient"] == "fd4") p.gradient = CONAN_GRAD_FD4;
    else if (C["gradient"] == "spectral") p.gradient = CONAN_GRAD_SPECTRAL;
    else throw Fail("gradient must be fd4 or spectral");
    p.periodic_gather = C.flag("periodic-gather");
    p.device = C.get<int>("device");
    conan_pm *h = conan_pm_create(&p);
    if (!h) throw Fail(conan_last_error());
    RunCtx ctx{H["id"], dim, N, L, format, (size_t)1};
    for (int k = 0; k < dim; ++k) ctx.np *= N;
    if (phi.size() != ctx.np) {
        conan_pm_destroy(h);
        throw Fail("potential record has the wrong size");
    }
    CbData cbd{&ctx};
    check(conan_pm_set_callback_interval(h, 10));
    int rc = conan_pm_run(h, phi.data(), a0, da, n, step_cb, &cbd);
    std::string msg = rc == CONAN_OK ? "" : (cbd.error.empty() ? conan_last_error() : cbd.error);
    try {
        ctx.join();  // the last snapshot's file
    } catch (std::exception &e) {
        if (msg.empty()) msg = e.what();
        rc = rc == CONAN_OK ? CONAN_ERR_IO : rc;
    }
    conan_pm_destroy(h);
    std::cout << std::endl;
    if (rc != CONAN_OK) throw Fail(msg);
}

// ---------------------------------------------------------------- cic ----

// The `cic` tool (src/cic/main.cc:11-82): density of snapshot <id>.pos.<m>
// on the (f N)^dim mesh, written as <id>.rho.<m>.conan.
void cmd_cic(int argc, char **argv) {
    Argv C;
    C.opts = {
        {0, "h", "help", "false", "print help on the use of this program."},
        {Option::VALUED | Option::CHECK, "i", "id", date_string(), "identifier for filenames."},
        {Option::VALUED | Option::CHECK, "f", "f", "2",
         "fractional Eulerian resolution. The default makes the Eulerian grid twice the size of the mass grid."},
        {Option::VALUED | Option::CHECK, "m", "m", "5", "snap-shot"},
        {Option::VALUED | Option::CHECK, "s", "sub-sample", "1", "subsample the grid and interpolate the position."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "device", "0", "CUDA device."},
    };
    C.parse(argc, argv);
    if (C.flag("help")) {
        std::cout << "Cosmic workset Conan (B200 build).\n\n";
        C.print(std::cout);
        exit(0);
    }
    unsigned m = C.get<unsigned>("m");
    std::ifstream fi(fmt(C["id"], ".pos.", m, ".conan"), std::ios::binary);
    if (!fi) throw Fail("Could not read from file");
    Header H;
    H.from_file(fi);
    H << C;
    History I;
    I.from_file(fi);
    I.update(C.command_line);
    unsigned f = H.get<unsigned>("f"), N = H.get<unsigned>("N");
    double L = H.get<double>("L");
    unsigned s = H.get<unsigned>("sub-sample");
    if (H.count("dim") == 0) H["dim"] = "3";
    int dim = H.get<int>("dim");
    std::vector<double> X = load_record(fi, "pos");
    fi.close();
    size_t np = 1;
    for (int k = 0; k < dim; ++k) np *= N;
    if (X.size() != np * (size_t)dim) throw Fail("pos record has the wrong size");

    conan_cic_params p{};
    p.dim = dim;
    p.n_mass = (int)N;
    p.f = (int)f;
    p.size = L;
    p.sub_sample = (int)s;
    p.device = C.get<int>("device");
    size_t nc = 1;
    for (int k = 0; k < dim; ++k) nc *= (size_t)N * f;
    std::vector<double> rho(nc);
    check(conan_cic(&p, X.data(), rho.data()));

    std::ofstream fo(fmt(C["id"], ".rho.", m, ".conan"), std::ios::binary);
    if (!fo) throw Fail("could not write the density file");
    H["N"] = fmt(N * f);
    H.to_file(fo);
    I.to_file(fo);
    save_record(fo, "density", "float64", rho.data(), rho.size() * sizeof(double));
}

// --------------------------------------------------------------- fof ----

// timed_filename (src/base/date.cc:34-49): <id>.<stage>.<round(b * 10^4), 5
// digits>.<ext>, or <id>.<stage>.init.<ext> for b < 0; b is a float.
std::string timed_filename(const std::string &id, const std::string &stage, float b, const std::string &ext) {
    std::ostringstream s;
    if (b < 0.0f)
        s << id << "." << stage << ".init" << ext;
    else
        s << id << "." << stage << "." << std::setfill('0') << std::setw(5) << static_cast<int>(std::round(b * 10000))
          << ext;
    return s.str();
}

// modulus(double, double), src/base/misc.hh:144-148.
double ref_modulus(double a, double b) {
    if (a < 0) return a - static_cast<int>(a / b - 1) * b;
    return a - static_cast<int>(a / b) * b;
}

// random_colour (src/fof/fof.cc:156-161): srand(t); rand() % 1022. glibc's
// rand() is random() on a 128-byte state; random_r on a private state of the
// same size gives the same numbers, so groups are coloured in parallel.
int group_colour(unsigned seed) {
    char state[128];
    struct random_data rd;
    std::memset(&rd, 0, sizeof rd);
    initstate_r(seed, state, sizeof state, &rd);
    int32_t r = 0;
    random_r(&rd, &r);
    return r % 1022;
}

// The text that fof_run writes after the header and history
// (src/fof/fof.cc:233-279): groups of at least 10 particles as "x y z  mass
// t" with the first (lowest-index) member's position wrapped by modulus, an
// empty line pair, then every group's members in index order as "x y z
// colour" with raw positions. Doubles print as std::ostream does (%g, 6
// digits). Formatting runs on all host threads in chunks written in order.
void write_fof(std::ostream &fo, int R, const std::vector<double> &X, const std::vector<unsigned long long> &tags,
               uint64_t ng, double L) {
    const size_t n = tags.size();
    std::vector<uint64_t> start(ng + 1, 0), first(ng, 0), order(n);
    for (size_t i = 0; i < n; ++i) {
        const uint64_t t = tags[i];
        if (t == 0 || t > ng) throw Fail("fof: group tag out of range");
        if (start[t] == 0) first[t - 1] = i;
        ++start[t];
    }
    for (uint64_t t = 0; t < ng; ++t) start[t + 1] += start[t];  // start[t] = first slot of group t (0-based)
    {
        std::vector<uint64_t> fill(start.begin(), start.end() - 1);
        for (size_t i = 0; i < n; ++i) order[fill[tags[i] - 1]++] = i;
    }
    unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
    std::vector<int> colour(ng);
    {
        std::vector<std::thread> th;
        for (unsigned w = 0; w < nt; ++w)
            th.emplace_back([&, w] {
                for (uint64_t t = w; t < ng; t += nt) colour[t] = group_colour((unsigned)t);
            });
        for (auto &t : th) t.join();
    }
    char buf[160];
    auto vec = [&](char *p, const double *x) {
        int k = 0;
        for (int a = 0; a < R; ++a) k += std::snprintf(p + k, sizeof buf - k, "%g ", x[a]);
        return k;
    };
    std::string head;
    for (uint64_t t = 0; t < ng; ++t) {
        const uint64_t m = start[t + 1] - start[t];
        if (m < 10) continue;
        double x[3];
        for (int a = 0; a < R; ++a) x[a] = ref_modulus(X[first[t] * R + a], L);
        int k = vec(buf, x);
        k += std::snprintf(buf + k, sizeof buf - k, " %llu %llu\n", (unsigned long long)m, (unsigned long long)t);
        head.append(buf, k);
    }
    head += "\n\n";
    fo << head;
    const size_t chunk = 1 << 20;
    for (size_t c0 = 0; c0 < n; c0 += chunk * nt) {
        std::vector<std::string> out(nt);
        std::vector<std::thread> th;
        for (unsigned w = 0; w < nt; ++w)
            th.emplace_back([&, w] {
                const size_t b = c0 + w * chunk, e = std::min(n, b + chunk);
                char lb[160];
                for (size_t s = b; s < e; ++s) {
                    const size_t i = order[s];
                    int k = 0;
                    for (int a = 0; a < R; ++a) k += std::snprintf(lb + k, sizeof lb - k, "%g ", X[i * R + a]);
                    k += std::snprintf(lb + k, sizeof lb - k, " %d\n", colour[tags[i] - 1]);
                    out[w].append(lb, k);
                }
            });
        for (auto &t : th) t.join();
        for (auto &o : out) fo << o;
    }
}

void cmd_fof(int argc, char **argv) {
    Argv C;
    C.opts = {
        {0, "h", "help", "false", "print help on the use of this program."},
        {Option::VALUED | Option::CHECK, "i", "id", date_string(), "identifier for filenames."},
        {Option::VALUED | Option::CHECK, "t", "time", "1.0", "time of snapshot."},
        {Option::VALUED | Option::CHECK, "l", "linking-length", "0.1", "linking length in units of Mpc h^-1."},
        {Option::VALUED | Option::CHECK, "f", "filename", "", "if given, supersedes internal naming system."},
        {0, "", "ascii", "true", "give output in ASCII."},
        {Option::VALUED | Option::CHECK | Option::LOCAL, "", "device", "0", "CUDA device."},
    };
    C.parse(argc, argv);
    if (C.flag("help")) {
        std::cout << "Cosmic workset Conan (B200 build).\n\n";
        C.print(std::cout);
        exit(0);
    }
    const double t = C.get<double>("time");
    const std::string fi_fn = C["filename"].empty() ? timed_filename(C["id"], "pos", (float)t, ".conan") : C["filename"];
    std::ifstream fi(fi_fn, std::ios::binary);
    if (!fi) throw Fail("Could not read from file " + fi_fn);
    Header H;
    H.from_file(fi);
    H << C;
    History I;
    I.from_file(fi);
    I.update(C.command_line);
    const int R = H.count("dim") == 1 ? H.get<int>("dim") : 3;
    const double L = H.get<double>("L"), ll = H.get<double>("linking-length");

    std::ofstream fo(timed_filename(C["id"], "fof", (float)t, ".txt"));
    if (!fo) throw Fail("could not write the fof file");
    fo << "# header\n";
    for (auto &kv : H) fo << "# " << kv.first << "=" << first_line(kv.second) << "\n";
    fo << "\n# history\n";
    for (auto &kv : I) fo << "# " << kv.first << ":" << first_line(kv.second) << "\n";
    fo << "\n";
    if (R != 2 && R != 3) return;  // fof_run exists for 2 and 3 dimensions only (src/fof/fof.cc:321-327)

    std::vector<double> X = load_record(fi, "pos");
    fi.close();
    const size_t n = X.size() / R;
    std::vector<unsigned long long> tags(n);
    unsigned long long ng = 0;
    conan_fof_params p{};
    p.dim = R;
    p.n_particles = n;
    p.size = L;
    p.linking_length = ll;
    p.device = C.get<int>("device");
    check(conan_fof(&p, X.data(), tags.data(), &ng));
    std::cerr << "[found " << ng << " groups]\n";
    write_fof(fo, R, X, tags, ng, L);
}

void usage(const std::string &cmd) {
    std::cout << "Conan - cosmological tool chain - NBody code (B200 build).\n\n"
                 "This is a very basic N-body code, using Particle-Mesh method.\n\n"
                 "usage: "
              << cmd << " [command] [args]\nwhere [command] is one of: ic, run, cic, fof\nto get help on a command: " << cmd
              << " [command] --help\n";
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) {
        usage(argv[0]);
        return 0;
    }
    std::map<std::string, std::function<void(int, char **)>> commands = {{"ic", cmd_ic}, {"run", cmd_run}, {"cic", cmd_cic}, {"fof", cmd_fof}};
    std::string command(argv[1]);
    try {
        auto it = commands.find(command);
        if (it == commands.end()) throw Fail("command [" + command + "] not understood.");
        it->second(argc - 1, argv + 1);
        return 0;
    } catch (std::exception &e) {
        std::cerr << "[error] " << e.what() << std::endl;
        usage(argv[0]);
        return 255;
    }
}

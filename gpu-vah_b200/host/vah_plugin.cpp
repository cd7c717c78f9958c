// vah_plugin.cpp -- the reference's driver surface over the C ABI: parameter
// loaders, .dat writer and the run() plugin (rhic/src/HydroPlugin.cpp:130-242,
// FileIO.cpp:14-59, {Lattice,Hydro,InitialCondition}Parameters.cpp).
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "vah.h"
#include "vah_plugin.h"
#include "vah_properties.h"

namespace {

constexpr double kHbarc = 0.197326938;
constexpr double kEosFactor = 13.8997;

bool load_file(const char *dir, const char *file, const char *what, vah::Properties *props) {
    char fname[512];
    std::snprintf(fname, sizeof(fname), "%s/%s", dir ? dir : "(null)", file);
    std::string err;
    if (!props->read_file(fname, &err)) {
        // LatticeParameters.cpp:25-28 (same wording)
        std::fprintf(stderr, "No configuration file  %s found for %s parameters - %s.\n", fname, what, err.c_str());
        std::fprintf(stderr, "Using default %s configuration parameters.\n", what);
        return false;
    }
    return true;
}

void get_int(const vah::Properties &p, const char *name, int *v, int dflt) {
    if (!p.lookup_int(name, v)) *v = dflt;
}

void get_double(const vah::Properties &p, const char *name, double *v, double dflt) {
    if (!p.lookup_float(name, v)) *v = dflt;
}

// Host-side EoS for the driver's printout and initial conditions
// (EquationOfState.cpp:31-201 conformal branch; table lookup as the kernels do).
struct HostEos {
    int kind = VAH_EOS_CONFORMAL;
    std::vector<double> tab;

    double pressure(double e) const {
        if (kind == VAH_EOS_CONFORMAL) return e / 3;
        return lookup(e, 0);
    }
    double temperature(double e) const {
        if (kind == VAH_EOS_CONFORMAL) return (double)powf((float)(e / kEosFactor), 0.25f);
        return lookup(e, 1);
    }
    double energy_density(double T) const {
        if (kind == VAH_EOS_CONFORMAL) return kEosFactor * powf((float)T, 4.0f);
        double lo = -60, hi = 60;
        for (int it = 0; it < 200; ++it) {
            double mid = 0.5 * (lo + hi);
            if (temperature(std::exp(mid)) < T) lo = mid; else hi = mid;
        }
        return std::exp(0.5 * (lo + hi));
    }
    double lookup(double e, int which) const {
        const int n = (int)tab[0];
        const double *v = tab.data() + 8 + (size_t)which * n;
        if (!(e > 0)) return which == 0 ? e * (tab[8] / tab[4]) : 0.0;
        const double x = std::log(e), f = (x - tab[1]) * tab[2];
        if (f <= 0) return which == 0 ? e * (v[0] / tab[4]) : v[0] * std::exp(3.0 / 23.0 * (x - tab[1]));
        if (f >= n - 1) return which == 0 ? e * (v[n - 1] / tab[6]) : v[n - 1] * std::exp(0.25 * (x - tab[5]));
        const int i = (int)f;
        const double w = f - i;
        return v[i] + w * (v[i + 1] - v[i]);
    }
};

int env_choice(const char *name, const char *const *options, int n, int dflt) {
    const char *v = std::getenv(name);
    if (!v) return dflt;
    for (int k = 0; k < n; ++k)
        if (std::strcmp(v, options[k]) == 0) return k;
    return dflt;
}

// Longitudinal profile of the reference's Glauber initial conditions
// (InitialConditions.cpp:196-215: eta_flat = 5.9, variance 0.16 hard-coded,
// eta = (k - (nz-1)/2) dz with integer division).
void reference_longitudinal(int nz, double dz, std::vector<double> &eL) {
    const double etaFlat = 5.9, etaVariance = 0.16;
    eL.resize(nz);
    for (int k = 0; k < nz; ++k) {
        const double eta = (k - (nz - 1) / 2) * dz;
        const double s = std::fabs(eta) - etaFlat / 2;
        const double arg = -s * s / etaVariance / 2 * (s < 0 ? 0.0 : 1.0);
        eL[k] = std::exp(arg);
    }
}

}  // namespace

extern "C" int vah_load_lattice_parameters(const char *dir, LatticeParameters *out) {
    vah::Properties p;
    const bool ok = load_file(dir, "lattice.properties", "lattice", &p);
    get_int(p, "numLatticePointsX", &out->numLatticePointsX, 128);
    get_int(p, "numLatticePointsY", &out->numLatticePointsY, 128);
    get_int(p, "numLatticePointsRapidity", &out->numLatticePointsRapidity, 64);
    get_int(p, "numProperTimePoints", &out->numProperTimePoints, 10);
    get_double(p, "latticeSpacingX", &out->latticeSpacingX, 0.08);
    get_double(p, "latticeSpacingY", &out->latticeSpacingY, 0.08);
    get_double(p, "latticeSpacingRapidity", &out->latticeSpacingRapidity, 0.3);
    get_double(p, "latticeSpacingProperTime", &out->latticeSpacingProperTime, 0.01);
    out->numComputationalLatticePointsX = out->numLatticePointsX + 4;
    out->numComputationalLatticePointsY = out->numLatticePointsY + 4;
    out->numComputationalLatticePointsRapidity = out->numLatticePointsRapidity + 4;
    return ok ? 0 : 1;
}

extern "C" int vah_load_initial_condition_parameters(const char *dir, InitialConditionParameters *out) {
    vah::Properties p;
    const bool ok = load_file(dir, "ic.properties", "initial condition", &p);
    get_int(p, "initialConditionType", &out->initialConditionType, 2);
    get_int(p, "numberOfNucleonsPerNuclei", &out->numberOfNucleonsPerNuclei, 208);
    get_double(p, "initialEnergyDensity", &out->initialEnergyDensity, 1.0);
    get_double(p, "scatteringCrossSectionNN", &out->scatteringCrossSectionNN, 62);
    get_double(p, "impactParameter", &out->impactParameter, 7);
    get_double(p, "fractionOfBinaryCollisions", &out->fractionOfBinaryCollisions, 0.5);
    get_double(p, "rapidityVariance", &out->rapidityVariance, 0.5);
    get_double(p, "rapidityMean", &out->rapidityMean, 0.5);
    return ok ? 0 : 1;
}

extern "C" int vah_load_hydro_parameters(const char *dir, HydroParameters *out) {
    vah::Properties p;
    const bool ok = load_file(dir, "hydro.properties", "hydrodynamic", &p);
    get_double(p, "initialProperTimePoint", &out->initialProperTimePoint, 0.1);
    get_double(p, "shearViscosityToEntropyDensity", &out->shearViscosityToEntropyDensity, 0.0795775);
    get_double(p, "freezeoutTemperatureGeV", &out->freezeoutTemperatureGeV, 0.155);
    get_int(p, "initializePimunuNavierStokes", &out->initializePimunuNavierStokes, 1);
    return ok ? 0 : 1;
}

extern "C" int vah_output(const double *var, double t, const char *dir, const char *name,
                          const LatticeParameters *lattice) {
    char fname[1024];
    std::snprintf(fname, sizeof(fname), "%s/%s_%.3f.dat", dir, name, t);
    FILE *fp = std::fopen(fname, "w");
    if (!fp) return -1;
    const int nx = lattice->numLatticePointsX, ny = lattice->numLatticePointsY, nz = lattice->numLatticePointsRapidity;
    const double dx = lattice->latticeSpacingX, dy = lattice->latticeSpacingY, dz = lattice->latticeSpacingRapidity;
    for (int k = 2; k < nz + 2; ++k) {
        const double z = (k - 2 - (nz - 1) / 2.) * dz;
        for (int j = 2; j < ny + 2; ++j) {
            const double y = (j - 2 - (ny - 1) / 2.) * dy;
            for (int i = 2; i < nx + 2; ++i) {
                const double x = (i - 2 - (nx - 1) / 2.) * dx;
                const size_t s = i + (size_t)(nx + 4) * (j + (size_t)(ny + 4) * k);
                std::fprintf(fp, "%.3f\t%.3f\t%.3f\t%.8f\n", x, y, z, var[s]);
            }
        }
    }
    std::fclose(fp);
    return 0;
}

namespace {

// Writes .dat snapshots on a thread of its own, so that formatting and file
// output (the bulk of an output step's cost) overlap the following GPU steps.
// The time loop copies each field to host memory (one synchronous copy) and
// queues it; jobs are written in the order queued. Queued data is bounded:
// push() waits while more than max_bytes are pending.
class DatWriter {
  public:
    DatWriter(const char *dir, const LatticeParameters &lat, size_t max_bytes)
        : dir_(dir ? dir : ""), lat_(lat), max_bytes_(max_bytes), thread_([this] { run(); }) {}
    ~DatWriter() { finish(); }

    void push(const char *name, double t, std::vector<double> &&data) {
        std::unique_lock<std::mutex> lock(mu_);
        space_.wait(lock, [&] { return pending_ == 0 || pending_ + data.size() * sizeof(double) <= max_bytes_; });
        pending_ += data.size() * sizeof(double);
        jobs_.push_back(Job{name, t, std::move(data)});
        ready_.notify_one();
    }

    // Waits for every queued file; returns the number that could not be written.
    int finish() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            if (done_) return failures_;
            done_ = true;
            ready_.notify_one();
        }
        thread_.join();
        return failures_;
    }

  private:
    struct Job {
        std::string name;
        double t;
        std::vector<double> data;
    };
    void run() {
        for (;;) {
            Job job;
            {
                std::unique_lock<std::mutex> lock(mu_);
                ready_.wait(lock, [&] { return done_ || !jobs_.empty(); });
                if (jobs_.empty()) return;
                job = std::move(jobs_.front());
                jobs_.pop_front();
            }
            if (vah_output(job.data.data(), job.t, dir_.c_str(), job.name.c_str(), &lat_) != 0) {
                std::fprintf(stderr, "cannot write %s/%s_%.3f.dat\n", dir_.c_str(), job.name.c_str(), job.t);
                ++failures_;
            }
            std::lock_guard<std::mutex> lock(mu_);
            pending_ -= job.data.size() * sizeof(double);
            space_.notify_all();
        }
    }
    std::string dir_;
    LatticeParameters lat_;
    size_t max_bytes_, pending_ = 0;
    std::deque<Job> jobs_;
    std::mutex mu_;
    std::condition_variable ready_, space_;
    bool done_ = false;
    int failures_ = 0;
    std::thread thread_;  // last: starts after the members it uses
};

// File names of the validity fields, as the reference's (commented-out)
// outputs name them (HydroPlugin.cpp:48-105), in VAH_V_* order.
const char *const kValidityNames[VAH_NUM_VALIDITY] = {
    "knTaupiT", "knTaupiL", "knTaupi", "knTauPi", "Rpi", "RPi", "Rpi2", "RPi2", "taupi",
    "dxux", "dyuy", "theta", "stt", "sxx", "syy", "snn", "regulations", "regMag",
    "regTr", "regU0", "regU1", "regU2", "regU3", "regZ0", "regZ1", "regZ2", "regZ3"};

}  // namespace

extern "C" int vah_run_plugin(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
                              const char *outputDir) {
    (void)rootDirectory;
    const LatticeParameters *lat = (const LatticeParameters *)latticeParams;
    const InitialConditionParameters *ic = (const InitialConditionParameters *)initCondParams;
    const HydroParameters *hydro = (const HydroParameters *)hydroParams;
    static const char *phys_names[] = {"ideal", "pimunu", "pimunu_pi"};
    static const char *eos_names[] = {"conformal", "table"};
    const int physics = env_choice("VAH_PHYSICS", phys_names, 3, VAH_PIMUNU);
    HostEos eos;
    eos.kind = env_choice("VAH_EOS", eos_names, 2, VAH_EOS_CONFORMAL);
    const int device = std::getenv("VAH_DEVICE") ? std::atoi(std::getenv("VAH_DEVICE")) : 0;
    if (eos.kind == VAH_EOS_TABLE) {
        eos.tab.assign(VAH_EOS_TABLE_LEN(VAH_EOS_TABLE_N), 0.0);
        int rc = vah_eos_table_build(VAH_EOS_TABLE_N, eos.tab.data(), eos.tab.size());
        if (rc != VAH_OK) return rc;
    }

    const int nt = lat->numProperTimePoints;
    const int nx = lat->numLatticePointsX, ny = lat->numLatticePointsY, nz = lat->numLatticePointsRapidity;
    const int ncx = nx + 4, ncy = ny + 4, ncz = nz + 4;
    const double t0 = hydro->initialProperTimePoint, dt = lat->latticeSpacingProperTime;
    const double dx = lat->latticeSpacingX, dy = lat->latticeSpacingY, dz = lat->latticeSpacingRapidity;
    const double Tf = hydro->freezeoutTemperatureGeV / kHbarc;
    std::printf("Grid size = %d x %d x %d\n", nx, ny, nz);
    std::printf("spatial resolution = (%.3f, %.3f, %.3f)\n", dx, dy, dz);
    std::printf("Grid size [fm] = %.3f x %.3f x %.3f\n", (nx - 1) / 2 * dx, (ny - 1) / 2 * dy, (nz - 1) / 2 * dz);
    std::printf("freezeout temperature = %.3f [fm^-1] (eF = %.3f [fm^-4])\n", Tf, eos.energy_density(Tf));
    std::printf(eos.kind == VAH_EOS_CONFORMAL ? "Using conformal EOS: e=3p.\n" : "Using QCD EOS.\n");
    std::printf("eta/s = %.6f\n", hydro->shearViscosityToEntropyDensity);

    vah_lattice vl{nx, ny, nz, dx, dy, dz};
    vah_hydro vh{t0, hydro->shearViscosityToEntropyDensity, hydro->freezeoutTemperatureGeV};
    static const char *precision_names[] = {"fp64", "fp32"};  // the FP64 form (default) or the FP32 form
    const int precision = env_choice("VAH_PRECISION", precision_names, 2, VAH_FP64);
    vah_options vo{physics, eos.kind, eos.kind == VAH_EOS_TABLE ? VAH_ZETA_CROSSOVER : VAH_ZETA_REFERENCE,
                   precision, VAH_FLUX_PER_CELL, device, nullptr};
    vah_event *ev = nullptr;
    int rc = vah_event_create(&vl, &vh, &vo, eos.kind == VAH_EOS_TABLE ? eos.tab.data() : nullptr, &ev);
    if (rc != VAH_OK) return rc;

    // initial conditions (InitialConditions.cpp:419-455)
    std::printf("Setting initial conditions: ");
    std::vector<double> e((size_t)nx * ny * nz), exy((size_t)nx * ny), eL;
    reference_longitudinal(nz, dz, eL);
    switch (ic->initialConditionType) {
    case 0: {
        std::printf("constant energy density.\n");
        const double ed = eos.energy_density(3.05);
        for (double &v : e) v = ed;
        break;
    }
    case 2:
    case 4: {
        const int A = ic->numberOfNucleonsPerNuclei;
        const double R = 1.12 * std::pow(A, 1. / 3.) - 0.86 * std::pow(A, -1. / 3.);
        const double sigma = 0.1 * ic->scatteringCrossSectionNN;  // mb -> fm^2
        const double e0 = eos.energy_density(ic->initialConditionType == 2 ? 3.05 : 2.03);
        if (ic->initialConditionType == 2) {
            std::printf("Continous optical Glauber.\n");
            rc = vah_ic_optical_glauber(nx, ny, dx, dy, ic->impactParameter, sigma, A, R, 0.54,
                                        ic->fractionOfBinaryCollisions, e0, 0.0, exy.data());
        } else {
            std::printf("Monte carlo Glauber.\n");
            rc = vah_ic_mc_glauber(nx, ny, dx, dy, ic->impactParameter, sigma, A, R, 0.54, 0.46, 1328398221ull, e0,
                                   0.0, exy.data(), nullptr);
        }
        if (rc != VAH_OK) break;
        for (int k = 0; k < nz; ++k)
            for (size_t s = 0; s < exy.size(); ++s) e[s + exy.size() * k] = exy[s] * eL[k] + 1.e-3;
        break;
    }
    default:
        std::printf("Initial condition type not defined. Exiting ...\n");
        rc = VAH_ERR_ARG;
    }
    if (rc == VAH_OK) {
        if (hydro->initializePimunuNavierStokes == 1)
            std::printf("Initialize \\pi^\\mu\\nu to its asymptotic Navier-Stokes value.\n");
        else
            std::printf("Initialize \\pi^\\mu\\nu to zero.\n");
        rc = vah_event_init_from_e(ev, t0, e.data(), VAH_PL_REFERENCE);
    }
    if (rc != VAH_OK) {
        vah_event_destroy(ev);
        return rc;
    }

    const int ictr = (nx % 2 == 0) ? ncx / 2 : (ncx - 1) / 2;
    const int jctr = (ny % 2 == 0) ? ncy / 2 : (ncy - 1) / 2;
    const int kctr = (nz % 2 == 0) ? ncz / 2 : (ncz - 1) / 2;
    const size_t sctr = ictr + (size_t)ncx * (jctr + (size_t)ncy * kctr);
    const size_t ncell = (size_t)ncx * ncy * ncz;
    std::vector<double> ebuf(ncell), pbuf(ncell);

    struct Out {
        int id;
        const char *name;
    };
    std::vector<Out> outs = {{VAH_F_E, "e"}, {VAH_F_P, "p"}, {VAH_F_UX, "ux"}, {VAH_F_UY, "uy"},
                             {VAH_F_UN, "un"}, {VAH_F_UT, "ut"}, {VAH_F_PL, "pl"}};
    if (physics != VAH_IDEAL) {
        const Out pis[] = {{VAH_F_PIXX, "pixx"}, {VAH_F_PIXY, "pixy"}, {VAH_F_PIXN, "pixn"}, {VAH_F_PIYY, "piyy"},
                           {VAH_F_PIYN, "piyn"}, {VAH_F_PITT, "pitt"}, {VAH_F_PITX, "pitx"}, {VAH_F_PITY, "pity"},
                           {VAH_F_PITN, "pitn"}, {VAH_F_PINN, "pinn"}};
        outs.insert(outs.end(), pis, pis + 10);
    }
    if (physics == VAH_PIMUNU_PI) outs.push_back({VAH_F_PI, "Pi"});
    // VAH_VALIDITY=1: also compute the validity diagnostics every step (as the
    // reference does) and write them with the other outputs
    const char *venv = std::getenv("VAH_VALIDITY");
    const bool validity = venv && std::atoi(venv) != 0;
    if (validity && (rc = vah_event_set_validity(ev, 1)) != VAH_OK) {
        vah_event_destroy(ev);
        return rc;
    }
    DatWriter writer(outputDir, *lat, (size_t)2 * (outs.size() + (validity ? VAH_NUM_VALIDITY : 0)) * ncell *
                                          sizeof(double));

    double t = t0, total_ms = 0;
    int nsteps = 0;
    for (int n = 1; n <= nt + 1 && rc == VAH_OK; ++n) {
        if ((n - 1) % 10 == 0) {  // FREQ, HydroPlugin.cpp:32,210-220
            if ((rc = vah_event_get_field(ev, VAH_F_E, ebuf.data(), 1)) != VAH_OK) break;
            if ((rc = vah_event_get_field(ev, VAH_F_P, pbuf.data(), 1)) != VAH_OK) break;
            std::printf("n = %d:%d (t = %.3f),\t (e, p) = (%.3f, %.3f) [GeV/fm^3],\t (T = %.3f [GeV]),\t", n - 1, nt,
                        t, ebuf[sctr] * kHbarc, pbuf[sctr] * kHbarc, eos.temperature(ebuf[sctr]) * kHbarc);
            for (const Out &o : outs) {
                std::vector<double> snap(ncell);
                if ((rc = vah_event_get_field(ev, o.id, snap.data(), 1)) != VAH_OK) break;
                if (outputDir) writer.push(o.name, t, std::move(snap));
            }
            for (int v = 0; validity && rc == VAH_OK && v < VAH_NUM_VALIDITY; ++v) {
                std::vector<double> snap(ncell);
                if ((rc = vah_event_get_validity(ev, v, snap.data(), 1)) != VAH_OK) break;
                if (outputDir) writer.push(kValidityNames[v], t, std::move(snap));
            }
            if (rc != VAH_OK) break;
        }
        auto a = std::chrono::steady_clock::now();
        rc = vah_rk2_step(ev, t, dt);
        if (rc == VAH_OK) rc = vah_event_sync(ev);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
        if ((n - 1) % 10 == 0) std::printf("(Elapsed time/step: %.3f ms)\n", ms);
        total_ms += ms;
        ++nsteps;
        t = t0 + n * dt;
    }
    if (nsteps) std::printf("Average time/step: %.3f ms\n", total_ms / nsteps);
    if (rc == VAH_ERR_NAN) std::printf("found NaN in the evolution (reference: exit(-1)).\n");
    writer.finish();  // every queued .dat file is on disk before run() returns
    vah_event_destroy(ev);
    return rc;
}

void run(void *latticeParams, void *initCondParams, void *hydroParams, const char *rootDirectory,
         const char *outputDir) {
    int rc = vah_run_plugin(latticeParams, initCondParams, hydroParams, rootDirectory, outputDir);
    if (rc != VAH_OK) std::fprintf(stderr, "run: libvah error %d\n", rc);
}

// vah_serve.cpp -- continuous-batching request loop over a vah_batch.
//
// Requests arrive as an open-loop Poisson stream (seeded). Each request's
// initial condition (MC-Glauber transverse profile, times the longitudinal
// profile for 3+1D) is built on a pool of host worker threads as soon as the
// request arrives. The driving thread admits built requests in arrival order
// while the batch has room (device footprint), advances every resident event
// in chunks of graph-replayed steps, and after each chunk reads the per-event
// maximum energy density (FP64 device reduction): an event whose maximum
// temperature fell below the freeze-out temperature is retired and its
// latency (arrival to retirement, wall clock) recorded. Work of events that
// arrive while others run overlaps with theirs on the device: they join the
// next chunk.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "vah.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    int id = 0;
    double arrival = 0;  // s after start
    vah_lattice lat{};
    double b = 0;
    unsigned long long seed = 0;
    std::vector<double> e;  // interior energy density, filled by a worker
    bool ready = false;
};

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

// e at which the table's temperature equals T (monotone table, bisection in ln e).
double energy_at_temperature(const std::vector<double> &tab, int eos, double T) {
    if (eos == VAH_EOS_CONFORMAL) return 13.8997 * std::pow(T, 4.0);
    const int n = (int)tab[0];
    const double *Tt = tab.data() + 8 + n;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) / 2;
        if (Tt[mid] < T) lo = mid; else hi = mid;
    }
    const double w = (T - Tt[lo]) / (Tt[hi] - Tt[lo]);
    return std::exp(tab[1] + tab[3] * (lo + w));
}

}  // namespace

extern "C" int vah_serve_run(const vah_serve_config *cfg, vah_serve_result *res, double *latencies,
                             int max_latencies) {
    if (!cfg || !res || cfg->rate <= 0 || cfg->duration_s <= 0 || cfg->chunk_steps < 1 || !(cfg->e_floor >= 0))
        return VAH_ERR_ARG;
    std::vector<double> tab;
    if (cfg->eos == VAH_EOS_TABLE) {
        tab.assign(VAH_EOS_TABLE_LEN(VAH_EOS_TABLE_N), 0.0);
        int rc = vah_eos_table_build(VAH_EOS_TABLE_N, tab.data(), tab.size());
        if (rc != VAH_OK) return rc;
    }
    vah_options opt{cfg->physics, cfg->eos, cfg->eos == VAH_EOS_TABLE ? VAH_ZETA_CROSSOVER : VAH_ZETA_REFERENCE,
                    cfg->precision, cfg->flux, cfg->device, nullptr};
    vah_batch *batch = nullptr;
    int rc = vah_batch_create(&opt, tab.empty() ? nullptr : tab.data(), cfg->capacity_bytes, &batch);
    if (rc != VAH_OK) return rc;

    // the request stream
    std::mt19937_64 rng(cfg->seed);
    std::exponential_distribution<double> gap(cfg->rate);
    std::uniform_real_distribution<double> unif(0.0, 1.0);
    std::vector<Request> reqs;
    for (double t = gap(rng); t < cfg->duration_s; t += gap(rng)) {
        Request r;
        r.id = (int)reqs.size();
        r.arrival = t;
        const bool is3d = unif(rng) < cfg->frac_3d;
        if (is3d) {
            const double f = unif(rng);  // linear between the smallest and largest 3D grid
            const int side = cfg->side3_min + (int)std::lround(f * (cfg->side3_max - cfg->side3_min));
            const int nz = cfg->nz3_min + (int)std::lround(f * (cfg->nz3_max - cfg->nz3_min));
            r.lat = {side, side, nz, cfg->dx, cfg->dx, cfg->deta};
        } else {
            const int side = cfg->side2_min + (int)(unif(rng) * (cfg->side2_max - cfg->side2_min + 1));
            r.lat = {side, side, 1, cfg->dx, cfg->dx, cfg->deta};
        }
        r.b = cfg->b_max * unif(rng);
        r.seed = rng();
        reqs.push_back(std::move(r));
    }
    const double T0fm = cfg->T0_GeV / 0.197326938, Tffm = cfg->Tf_GeV / 0.197326938;
    const double e_peak = energy_at_temperature(tab, cfg->eos, T0fm);
    const double e_freeze = energy_at_temperature(tab, cfg->eos, Tffm);

    // IC workers: build each request's e as soon as it has arrived
    const auto t_start = Clock::now();
    std::mutex mu;
    std::condition_variable cv;
    std::atomic<int> next_build{0};
    std::atomic<bool> stop{false};
    auto worker = [&]() {
        if (cfg->ic_on_device) return;  // the IC is generated at admission
        for (;;) {
            const int k = next_build.fetch_add(1);
            if (k >= (int)reqs.size() || stop) return;
            Request &r = reqs[k];
            const double wait = r.arrival - seconds_since(t_start);
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
            std::vector<double> exy((size_t)r.lat.nx * r.lat.ny), f(r.lat.nz), e((size_t)r.lat.nx * r.lat.ny * r.lat.nz);
            vah_ic_mc_glauber(r.lat.nx, r.lat.ny, r.lat.dx, r.lat.dy, r.b, 4.2, 197, 6.38, 0.535, 0.5, r.seed, e_peak,
                              0.0, exy.data(), nullptr);
            vah_ic_longitudinal(r.lat.nz, r.lat.dz, 1.5, 1.3, f.data());
            // the floor goes on after the product, as InitialConditions.cpp:247 adds it
            for (int k2 = 0; k2 < r.lat.nz; ++k2)
                for (size_t s = 0; s < exy.size(); ++s) e[s + exy.size() * k2] = exy[s] * f[k2] + cfg->e_floor;
            std::lock_guard<std::mutex> lock(mu);
            r.e = std::move(e);
            r.ready = true;
            cv.notify_one();
        }
    };
    const int nworkers = std::max(1, std::min(cfg->ic_threads, 64));
    std::vector<std::thread> pool;
    for (int w = 0; w < nworkers; ++w) pool.emplace_back(worker);

    struct Live {
        int req, slot;
    };
    std::vector<Live> live;
    std::vector<double> lat_s;
    std::vector<int> queue_order;  // arrived requests, arrival order
    int next_admit = 0;            // requests admitted or refused so far, in arrival order
    long long cell_updates = 0, chunk_count = 0, max_resident = 0, timeouts = 0, rejected = 0, failed = 0;
    double last_done = 0, tau_freeze_max = 0;
    std::vector<double> emax;
    rc = VAH_OK;
    while (rc == VAH_OK) {
        // admit built requests in arrival order while there is room
        bool refused = false;
        while (next_admit < (int)reqs.size() && !refused) {
            Request &r = reqs[next_admit];
            if (cfg->ic_on_device) {
                if (seconds_since(t_start) < r.arrival) break;
            } else {
                std::unique_lock<std::mutex> lock(mu);
                if (!r.ready) break;
            }
            vah_hydro hy{cfg->t0, cfg->eta_over_s, cfg->Tf_GeV};
            int slot = -1;
            int a;
            if (cfg->ic_on_device) {
                const vah_glauber g{r.b, 4.2, 197, 6.38, 0.535, 0.5, r.seed, e_peak, cfg->e_floor, 1.5, 1.3};
                a = vah_batch_add_glauber(batch, &r.lat, &hy, cfg->dt, &g, VAH_PL_ISOTROPIC, &slot);
            } else {
                a = vah_batch_add(batch, &r.lat, &hy, cfg->dt, r.e.data(), VAH_PL_ISOTROPIC, &slot);
            }
            if (a == VAH_ERR_FULL) {
                refused = live.empty() ? false : true;
                if (live.empty()) {  // larger than the whole batch: reject the request
                    ++rejected;
                    ++next_admit;
                }
                break;
            }
            if (a != VAH_OK) {
                rc = a;
                break;
            }
            std::vector<double>().swap(r.e);
            live.push_back({next_admit, slot});
            ++next_admit;
        }
        if (rc != VAH_OK) break;
        if (live.empty()) {
            if (next_admit >= (int)reqs.size()) break;
            std::unique_lock<std::mutex> lock(mu);
            cv.wait_for(lock, std::chrono::milliseconds(5));
            continue;
        }
        max_resident = std::max<long long>(max_resident, (long long)live.size());
        long long chunk_cells = 0;
        for (const Live &l : live) {
            const vah_lattice &L = reqs[l.req].lat;
            chunk_cells += (long long)L.nx * L.ny * L.nz;
        }
        if ((rc = vah_batch_step(batch, cfg->chunk_steps)) != VAH_OK) break;
        cell_updates += chunk_cells * cfg->chunk_steps;
        ++chunk_count;
        int maxslot = 0;
        for (const Live &l : live) maxslot = std::max(maxslot, l.slot);
        emax.assign(maxslot + 1, 0.0);
        if ((rc = vah_batch_max_energy_density(batch, emax.data(), maxslot + 1)) != VAH_OK) break;
        std::vector<Live> keep;
        for (const Live &l : live) {
            vah_event_info info;
            vah_batch_event_info(batch, l.slot, &info);
            const bool frozen = info.nan_cells == 0 && emax[l.slot] < e_freeze;
            const bool too_old = info.t > cfg->t_max;
            if (frozen || too_old || info.nan_cells > 0) {
                const double now = seconds_since(t_start);
                if (frozen) {  // latency statistics cover events that reached freeze-out
                    lat_s.push_back(now - reqs[l.req].arrival);
                    last_done = now;
                    tau_freeze_max = std::max(tau_freeze_max, info.t);
                } else {
                    ++timeouts;
                    if (info.nan_cells > 0) ++failed;
                }
                vah_batch_remove(batch, l.slot);
            } else {
                keep.push_back(l);
            }
        }
        live.swap(keep);
    }
    stop = true;
    for (auto &t : pool) t.join();
    vah_batch_destroy(batch);
    if (rc != VAH_OK) return rc;

    std::vector<double> sorted = lat_s;
    std::sort(sorted.begin(), sorted.end());
    auto pct = [&](double q) {
        if (sorted.empty()) return 0.0;
        const size_t k = (size_t)std::min<double>(sorted.size() - 1, std::floor(q * (sorted.size() - 1) + 0.5));
        return sorted[k];
    };
    res->offered = (long long)reqs.size();
    res->completed = (long long)lat_s.size();
    res->timeouts = timeouts;
    res->rejected = rejected;
    res->wall_s = seconds_since(t_start);
    res->events_per_s = last_done > 0 ? lat_s.size() / last_done : 0.0;
    res->p50_s = pct(0.50);
    res->p99_s = pct(0.99);
    res->cell_updates = cell_updates;
    res->cell_updates_per_s = res->wall_s > 0 ? cell_updates / res->wall_s : 0.0;
    res->max_resident = max_resident;
    res->chunks = chunk_count;
    res->failed = failed;
    res->tau_freeze_max = tau_freeze_max;
    if (latencies)
        for (int k = 0; k < max_latencies && k < (int)lat_s.size(); ++k) latencies[k] = lat_s[k];
    return VAH_OK;
}

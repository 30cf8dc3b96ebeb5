// server.cpp — a request loop serving R/T spectrum jobs with continuous batching.
//
// Jobs (normal-incidence unit cells: grid, structure map, materials, pulse,
// step budget) are submitted at any time and wait in a host queue that holds
// no device memory. Each poll:
//  1. retires the members that used up their budget: their R/T spectra are
//     computed (aefdtd_get_normal_spectra), their simulations destroyed and
//     their device memory returned to the budget;
//  2. admits queued jobs in arrival order (looking past at most `lookahead`
//     jobs that do not fit) while the estimated device footprint of each fits
//     the memory budget (by default 80% of the device's HBM) and the number of
//     running jobs is below max_active: the simulation is created and set up on
//     the device and joins the batch with its step budget;
//  3. advances the batch by one segment (at most segment_steps steps; a subset
//     stops early when one of its members finishes).
// So requests that arrive while others run join between segments, share the
// merged launches of their size class, and leave as soon as they are done.
// Fields and plane sums stay resident on the device from admission to
// retirement. Every job's submit, admit and done times are kept; the stats
// give p50/p99 time-to-spectrum (submit -> done), sims/s and cell-updates/s.
//
// Results do not depend on the mix: a member computes exactly what it would
// compute as the only member (same kernels, same arithmetic per cell).
#include "sim.hpp"

#include <chrono>
#include <deque>

namespace aefdtd {

struct Job {
    int id = 0;
    int state = 0;   // AEFDTD_JOB_*
    aefdtd_grid_desc g{};
    std::vector<uint32_t> map;
    std::vector<aefdtd_material_desc> mats;
    aefdtd_normal_desc nd{};
    int steps = 0;
    double cc_coeff = 0;
    int cc_step = 500, stop = -1;
    size_t est = 0, bytes = 0;
    long long cells = 0;
    aefdtd_sim *sim = nullptr;
    double t_submit = 0, t_admit = -1, t_done = -1;
    std::vector<double> spectra;
    std::string error;
};

// Device bytes a job will hold, from the same sizing rules as the simulation
// constructor (total grid, CPML slabs, recursive-convolution boxes, plane-sum
// history, work lists), with a 10% margin. No device call.
size_t estimate_job_bytes(const Job &j) {
    const aefdtd_grid_desc &g = j.g;
    int pml[6], pad[6];
    for (int f = 0; f < 6; f++) { pml[f] = std::max(0, g.pml[f]); pad[f] = std::max(0, g.pad[f]); }
    if (g.mode == AEFDTD_MODE_NORMAL) {
        for (int f = 0; f < 4; f++) { pml[f] = 0; pad[f] = 0; }
        pad[4] = std::max(5, pad[4]);
        pad[5] = std::max(5, pad[5]);
    } else {
        for (int a = 0; a < 3; a++)
            if (pml[2 * a] || pml[2 * a + 1]) {
                pad[2 * a] = std::max(5, pad[2 * a]);
                pad[2 * a + 1] = std::max(5, pad[2 * a + 1]);
            }
    }
    const size_t Nx = g.nx + pml[0] + pad[0] + pad[1] + pml[1];
    const size_t Ny = g.ny + pml[2] + pad[2] + pad[3] + pml[3];
    const size_t Nz = g.nz + pml[4] + pad[4] + pad[5] + pml[5];
    const size_t N = Nx * Ny * Nz, es = g.precision == AEFDTD_FP64 ? 8 : 4;
    const size_t idb = j.mats.size() <= 256 ? 1 : 2;
    size_t b = 6 * N * es;                                                 // fields
    b += ((Nx * idb + 15) / 16 * 16) * Ny * Nz;                            // material ids (pitched)
    const size_t nxs = pml[0] + pml[1], nys = pml[2] + pml[3], nzs = pml[4] + pml[5];
    b += 4 * (nxs * Ny * Nz + Nx * nys * Nz + Nx * Ny * nzs) * es;         // CPML psi, E and H
    // recursive-convolution psi: bounding box of each dispersive material in
    // the structure map, extended to the grid edge where the map touches it
    // (edge slices are replicated into pads and PML)
    size_t rc = 0;   // recursive-convolution psi
    for (size_t m = 0; m < j.mats.size(); m++) {
        const aefdtd_material_desc &md = j.mats[m];
        const int np = md.n_debye + md.n_drude + md.n_lorentz + md.n_critpoint;
        if (np <= 0) continue;
        int x1 = g.nx, x2 = -1, y1 = g.ny, y2 = -1, z1 = g.nz, z2 = -1;
        for (int k = 0; k < g.nz; k++)
            for (int jy = 0; jy < g.ny; jy++)
                for (int i = 0; i < g.nx; i++)
                    if (j.map[i + size_t(g.nx) * (jy + size_t(g.ny) * k)] == m) {
                        x1 = std::min(x1, i); x2 = std::max(x2, i);
                        y1 = std::min(y1, jy); y2 = std::max(y2, jy);
                        z1 = std::min(z1, k); z2 = std::max(z2, k);
                    }
        if (x2 < 0) continue;
        const size_t bx = (x1 == 0 ? pml[0] + pad[0] : 0) + (x2 == g.nx - 1 ? pml[1] + pad[1] : 0) + (x2 - x1 + 1);
        const size_t by = (y1 == 0 ? pml[2] + pad[2] : 0) + (y2 == g.ny - 1 ? pml[3] + pad[3] : 0) + (y2 - y1 + 1);
        const size_t bz = (z1 == 0 ? pml[4] + pad[4] : 0) + (z2 == g.nz - 1 ? pml[5] + pad[5] : 0) + (z2 - z1 + 1);
        b += bx * by * bz * 3 * size_t(np) * 2 * es;
        rc += bx * by * bz * 3 * size_t(np) * 2 * es;
    }
    // a job that runs alone in its subset takes the fused time step: a second
    // set of fields, E-side CPML psi and RC psi
    const char *fz = std::getenv("AEFDTD_FUSED");
    if (g.mode != AEFDTD_MODE_OBLIQUE && (fz ? atoi(fz) != 0 : kFusedDefault))
        b += 6 * N * es + 2 * (nxs * Ny * Nz + Nx * nys * Nz + Nx * Ny * nzs) * es + rc;
    const int seg = g.dft_block > 0 ? g.dft_block : 64;
    b += size_t(std::max(std::max(g.nt, j.steps), 1024)) * 12 * 8;        // plane-sum history
    b += size_t(seg) * kPlaneBlocks * 12 * 8;                               // plane-sum partials
    if (j.cc_coeff > 0) b += size_t(j.steps) * 8 + size_t(seg) * 2 * 148 * 8;  // completion energies
    b += N / 16 + 2 * sizeof(StepScalars) * seg + (1 << 16);                // work lists, tables, small
    return b + b / 10;
}

}  // namespace aefdtd

using namespace aefdtd;

struct aefdtd_server {
    std::string last_error;
    aefdtd_server_opts opts{};
    aefdtd_batch *batch = nullptr;
    std::vector<Job> jobs;
    std::deque<int> queue;
    std::map<aefdtd_sim *, int> running;   // simulation -> job
    size_t budget = 0, in_use = 0, peak = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
    int retire();
    void admit();
    ~aefdtd_server() {
        for (auto &kv : running) aefdtd_destroy(kv.first);
        if (batch) aefdtd_batch_destroy(batch);
    }
};

int aefdtd_server::retire() {
    int n = 0;
    if (aefdtd_batch_finished(batch, nullptr, 0, &n) != AEFDTD_OK) fail(AEFDTD_CUDA_ERROR, aefdtd_batch_last_error(batch));
    if (n == 0) return 0;
    std::vector<aefdtd_sim *> done(n);
    aefdtd_batch_finished(batch, done.data(), n, &n);
    for (aefdtd_sim *s : done) {
        Job &j = jobs[running.at(s)];
        j.spectra.assign(size_t(15) * j.nd.nl, 0.0);
        aefdtd_status st = aefdtd_get_normal_spectra(s, j.spectra.data(), j.nd.nl);
        j.t_done = now();
        if (j.cc_coeff > 0) {
            int32_t cdone = 0, cstop = -1;
            double ratio = 0;
            aefdtd_get_completion(s, &cdone, &cstop, &ratio);
            j.stop = cdone ? cstop : -1;
        }
        if (st == AEFDTD_OK) {
            j.state = AEFDTD_JOB_DONE;
        } else {
            j.state = AEFDTD_JOB_FAILED;
            j.error = aefdtd_last_error(s);
        }
        aefdtd_batch_remove(batch, s);
        aefdtd_destroy(s);
        in_use -= j.bytes;
        running.erase(s);
        j.sim = nullptr;
    }
    return n;
}

void aefdtd_server::admit() {
    int looked = 0;
    aefdtd_batch_info bi{};
    aefdtd_batch_get_info(batch, &bi);
    const size_t overhead = (size_t)bi.batch_bytes;   // the batch's work lists and argument arrays
    for (auto it = queue.begin(); it != queue.end();) {
        if (opts.max_active > 0 && (int)running.size() >= opts.max_active) break;
        Job &j = jobs[*it];
        if (j.est > budget) {
            j.state = AEFDTD_JOB_FAILED;
            j.error = "footprint above the memory budget";
            it = queue.erase(it);
            continue;
        }
        if (in_use + overhead + j.est > budget) {
            if (++looked > opts.lookahead) break;
            ++it;
            continue;
        }
        // create and set up on the device; any failure fails the job, not the server
        aefdtd_sim *s = nullptr;
        aefdtd_status st = aefdtd_create(&j.g, &s);
        if (st == AEFDTD_OK) st = aefdtd_set_material_map(s, j.map.data(), j.map.size());
        for (size_t m = 0; st == AEFDTD_OK && m < j.mats.size(); m++) st = aefdtd_set_material(s, (uint32_t)m, &j.mats[m]);
        if (st == AEFDTD_OK) st = aefdtd_setup_normal(s, &j.nd);
        if (st == AEFDTD_OK && j.cc_coeff > 0) st = aefdtd_set_completion(s, j.cc_coeff, j.cc_step);
        if (st == AEFDTD_OK && aefdtd_batch_add(batch, s, j.steps) != AEFDTD_OK) {
            st = AEFDTD_BAD_ARG;
            j.error = aefdtd_batch_last_error(batch);
        }
        if (st != AEFDTD_OK) {
            if (j.error.empty()) j.error = s ? aefdtd_last_error(s) : aefdtd_last_error(nullptr);
            if (s) aefdtd_destroy(s);
            j.state = AEFDTD_JOB_FAILED;
            it = queue.erase(it);
            continue;
        }
        aefdtd_dims d{};
        aefdtd_get_dims(s, &d);
        j.bytes = d.device_bytes;
        j.cells = (long long)d.nx * d.ny * d.nz;
        j.sim = s;
        j.state = AEFDTD_JOB_RUNNING;
        j.t_admit = now();
        in_use += j.bytes;
        peak = std::max(peak, in_use);
        running[s] = j.id;
        j.map.clear();
        j.map.shrink_to_fit();
        it = queue.erase(it);
    }
}

template <typename F> static aefdtd_status sguarded(aefdtd_server *v, F &&f) {
    try {
        f();
        if (v) v->last_error.clear();
        return AEFDTD_OK;
    } catch (Error &e) {
        if (v) v->last_error = e.msg;
        return e.st;
    } catch (std::bad_alloc &) {
        if (v) v->last_error = "host allocation failed";
        return AEFDTD_OOM;
    } catch (std::exception &e) {
        if (v) v->last_error = e.what();
        return AEFDTD_BAD_ARG;
    }
}

static double percentile(std::vector<double> v, double p) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    const double r = p * (v.size() - 1);
    const size_t lo = (size_t)r, hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (v[hi] - v[lo]) * (r - lo);
}

extern "C" {

aefdtd_status aefdtd_server_create(const aefdtd_server_opts *opts, aefdtd_server **out) {
    if (!out) return AEFDTD_BAD_ARG;
    *out = nullptr;
    auto *v = new aefdtd_server();
    aefdtd_status st = sguarded(v, [&] {
        if (opts) {
            if (opts->abi_version != AEFDTD_ABI_VERSION) fail(AEFDTD_BAD_ARG, "abi_version mismatch");
            v->opts = *opts;
        } else {
            v->opts.abi_version = AEFDTD_ABI_VERSION;
        }
        // defaults measured on a Poisson stream of 32 unit-cell jobs, 10% large cells
        // (the batch's L2-resident members without an up-front L2 prefetch, lanes
        // sized by subset bytes): 256 steps per poll and the batch's L2-sized
        // subsets (48 MiB) gave p50 1.6 s, p99 6.1 s, 45.6 Gcell/s, against 4.0 s,
        // 13.3 s, 38.5 Gcell/s for one merged subset per size class and 3.0 s,
        // 7.6 s, 44.0 Gcell/s for 64 steps per poll
        if (v->opts.segment_steps <= 0) v->opts.segment_steps = 256;
        if (v->opts.lookahead <= 0) v->opts.lookahead = 16;
        aefdtd_batch_opts bo = v->opts.batch;
        bo.abi_version = AEFDTD_ABI_VERSION;
        bo.device = v->opts.device;
        aefdtd_status b = aefdtd_batch_create(&bo, &v->batch);
        if (b != AEFDTD_OK) fail(b, "batch creation failed");
        size_t fr = 0, tot = 0;
        AE_CUDA(cudaSetDevice(v->opts.device));
        AE_CUDA(cudaMemGetInfo(&fr, &tot));
        const double frac = v->opts.hbm_fraction > 0 ? v->opts.hbm_fraction : 0.8;
        v->budget = v->opts.budget_bytes > 0 ? (size_t)v->opts.budget_bytes : (size_t)(frac * (double)tot);
    });
    if (st != AEFDTD_OK) {
        delete v;
        return st;
    }
    *out = v;
    return AEFDTD_OK;
}

aefdtd_status aefdtd_server_destroy(aefdtd_server *v) {
    if (!v) return AEFDTD_BAD_ARG;
    delete v;
    return AEFDTD_OK;
}

const char *aefdtd_server_last_error(const aefdtd_server *v) { return v ? v->last_error.c_str() : ""; }

aefdtd_status aefdtd_server_submit(aefdtd_server *v, const aefdtd_job_desc *jd, int32_t *job_id) {
    if (!v || !jd || !jd->grid || !jd->map || !jd->materials || !jd->normal) return AEFDTD_BAD_ARG;
    return sguarded(v, [&] {
        const aefdtd_grid_desc &g = *jd->grid;
        if (g.mode != AEFDTD_MODE_NORMAL) fail(AEFDTD_BAD_ARG, "served jobs are normal-incidence cells");
        if (g.nx < 1 || g.ny < 1 || g.nz < 1) fail(AEFDTD_BAD_ARG, "grid sizes must be positive");
        if (jd->map_count != size_t(g.nx) * g.ny * g.nz) fail(AEFDTD_BAD_ARG, "map size must be nx*ny*nz");
        if (jd->n_materials < 1 || jd->steps < 1 || jd->normal->nl < 1) fail(AEFDTD_BAD_ARG, "empty job");
        for (size_t i = 0; i < jd->map_count; i++)
            if (jd->map[i] >= (uint32_t)jd->n_materials) fail(AEFDTD_BAD_ARG, "map index without a material");
        Job j;
        j.id = (int)v->jobs.size();
        j.state = AEFDTD_JOB_QUEUED;
        j.g = g;
        j.g.device = v->opts.device;
        j.map.assign(jd->map, jd->map + jd->map_count);
        j.mats.assign(jd->materials, jd->materials + jd->n_materials);
        j.nd = *jd->normal;
        j.steps = jd->steps;
        if (!(jd->cc_coeff >= 0) || jd->cc_step < 0) fail(AEFDTD_BAD_ARG, "bad completion settings");
        j.cc_coeff = jd->cc_coeff;
        j.cc_step = jd->cc_step > 0 ? jd->cc_step : 500;
        j.est = estimate_job_bytes(j);
        j.t_submit = v->now();
        v->jobs.push_back(std::move(j));
        v->queue.push_back(v->jobs.back().id);
        if (job_id) *job_id = v->jobs.back().id;
    });
}

aefdtd_status aefdtd_server_poll(aefdtd_server *v, int32_t *n_done) {
    if (!v) return AEFDTD_BAD_ARG;
    return sguarded(v, [&] {
        int done = v->retire();
        v->admit();
        if (!v->running.empty()) {
            int32_t ran = 0;
            aefdtd_status st = aefdtd_batch_advance(v->batch, v->opts.segment_steps, &ran);
            if (st != AEFDTD_OK) fail(st, aefdtd_batch_last_error(v->batch));
            done += v->retire();
        }
        if (n_done) *n_done = done;
    });
}

aefdtd_status aefdtd_server_job_info(aefdtd_server *v, int32_t job, aefdtd_job_info *info) {
    if (!v || !info) return AEFDTD_BAD_ARG;
    return sguarded(v, [&] {
        if (job < 0 || job >= (int)v->jobs.size()) fail(AEFDTD_BAD_ARG, "unknown job");
        const Job &j = v->jobs[job];
        std::memset(info, 0, sizeof(*info));
        info->state = j.state;
        info->cells = j.cells;
        info->est_bytes = (int64_t)j.est;
        info->bytes = (int64_t)j.bytes;
        info->t_submit = j.t_submit;
        info->t_admit = j.t_admit;
        info->t_done = j.t_done;
        info->steps = j.steps;
        info->stop_step = j.stop;
    });
}

aefdtd_status aefdtd_server_job_spectra(aefdtd_server *v, int32_t job, double *out, int32_t nl) {
    if (!v || !out) return AEFDTD_BAD_ARG;
    return sguarded(v, [&] {
        if (job < 0 || job >= (int)v->jobs.size()) fail(AEFDTD_BAD_ARG, "unknown job");
        const Job &j = v->jobs[job];
        if (j.state == AEFDTD_JOB_FAILED) fail(AEFDTD_BAD_ARG, "job failed: " + j.error);
        if (j.state != AEFDTD_JOB_DONE) fail(AEFDTD_NOT_READY, "job not done");
        if (nl != j.nd.nl) fail(AEFDTD_BAD_ARG, "nl must equal the job's spectrum size");
        std::memcpy(out, j.spectra.data(), j.spectra.size() * sizeof(double));
    });
}

aefdtd_status aefdtd_server_get_stats(aefdtd_server *v, aefdtd_server_stats *st) {
    if (!v || !st) return AEFDTD_BAD_ARG;
    return sguarded(v, [&] {
        std::memset(st, 0, sizeof(*st));
        std::vector<double> lat;
        double first = 1e300, last = 0, cu = 0;
        for (const Job &j : v->jobs) {
            st->submitted++;
            if (j.state == AEFDTD_JOB_QUEUED) st->queued++;
            if (j.state == AEFDTD_JOB_RUNNING) st->running++;
            if (j.state == AEFDTD_JOB_FAILED) st->failed++;
            if (j.state == AEFDTD_JOB_DONE) {
                st->done++;
                lat.push_back(j.t_done - j.t_submit);
                first = std::min(first, j.t_submit);
                last = std::max(last, j.t_done);
                cu += double(j.cells) * j.steps;
            }
        }
        st->budget_bytes = (int64_t)v->budget;
        st->in_use_bytes = (int64_t)v->in_use;
        st->peak_bytes = (int64_t)v->peak;
        st->p50_s = percentile(lat, 0.50);
        st->p99_s = percentile(lat, 0.99);
        double sum = 0;
        for (double x : lat) sum += x;
        st->mean_s = lat.empty() ? 0 : sum / lat.size();
        st->elapsed_s = lat.empty() ? 0 : last - first;
        st->sims_per_s = st->elapsed_s > 0 ? st->done / st->elapsed_s : 0;
        st->gcells_per_s = st->elapsed_s > 0 ? cu / st->elapsed_s / 1e9 : 0;
    });
}

}  // extern "C"

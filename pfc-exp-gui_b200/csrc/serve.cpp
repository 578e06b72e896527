// serve.cpp -- the engine: Misfit / CVD runs and Elastic analyses submitted from any
// thread, admitted by device-memory budget and advanced together on one GPU.
//
// The reference runs one pfc-exp-cli process per parameter set, one after the other
// (src/gui/MainWindow.cpp:3453-3522, the sweep queue built at MainWindow.cpp:2632-2770).
// Here one scheduler thread owns the GPU:
//   * admission: queued jobs are admitted in submission order while their device bytes
//     (pfc_run_bytes) fit the budget and the active-run limit; a job that does not fit
//     waits, and so do the jobs behind it;
//   * continuous batching: active runs are grouped into cohorts of one model and grid;
//     every quantum advances all cohorts by the same number of steps, the regular steps
//     as one CUDA graph per composition (one stream per cohort, so small grids run side
//     by side), and jobs join or leave between quanta;
//   * checkpoints: a quantum ends at the nearest checkpoint of any active run.  Each run
//     takes exactly the kernel sequence of pfc_run_advance in the CLI (a Misfit
//     checkpoint step uses the checkpoint column mode; a CVD step always ends with the
//     energy analysis, CVD:442), so a job's fields, energies and files are the same
//     alone, in any mix and from pfc-exp-cli;
//   * output: results are copied to the host and handed to a writer thread, which
//     writes the pfc-exp-cli files (checkpoint.h) and then posts the job's events.
// CVD energies are kept per step on the device (launch_reduce_runs) and copied out
// asynchronously per graph segment, so the per-step energy.txt lines add no
// synchronisation inside a quantum.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "checkpoint.h"
#include "pfc_b200.h"
#include "pfc_engine.h"
#include "pfc_internal.h"

using namespace pfc;
using namespace pfc::ckpt;

namespace pfc {
cudaError_t launch_reduce_fixed(const double *partials, int count, int stride, int width, double *out,
                                cudaStream_t s);
}

namespace {

constexpr int SEG = 16;  // steps per captured graph segment (and CVD energy slots per run)

enum class State { Pending, Active, Done, Failed, Cancelled };

// What an event needs to know about its job (copied into writer tasks).
struct JobTimes {
    uint64_t id = 0;
    double t_submit = 0.0, t_admit = -1.0;
};

struct Job {
    uint64_t id = 0;
    pfc_job spec{};
    std::string outdir, input_dir;
    State state = State::Pending;
    bool cancel_req = false;
    double bytes = 0.0;
    double t_submit = 0.0, t_admit = -1.0;
    pfc_run *run = nullptr;
    int t = 0;  // steps taken
    // CVD: energy sums of the steps of the current quantum (host copy)
    std::vector<double> ehist;
    // final fields of a finished run (kept until pfc_release)
    std::shared_ptr<std::vector<float>> phi, con;
    int L = 0, M = 0, N = 1;
    JobTimes times() const { return JobTimes{id, t_submit, t_admit}; }
};

// Steps after which a Misfit run checkpoints: t % mod == 0 or t == steps (MIS:513).
bool misfit_ckpt(const Job &j, int t) { return t % j.spec.mod == 0 || t == j.spec.steps; }
// CVD writes its fields after step s = t + 1 when t % mod == 0 (CVD:425-438).
bool cvd_ckpt(const Job &j, int s) { return (s - 1) % j.spec.mod == 0; }

// Steps until the run's next event (a checkpoint or its end).
int steps_to_event(const Job &j) {
    for (int s = j.t + 1; s <= j.spec.steps; ++s) {
        if (s == j.spec.steps) return s - j.t;
        if (j.spec.kind == PFC_JOB_MISFIT ? misfit_ckpt(j, s) : cvd_ckpt(j, s)) return s - j.t;
    }
    return 0;
}

struct Cohort {
    int model = 0, L = 0, M = 0, CT = 0, stage = 0, prec = 0;  // runs of one model, grid, tile width, staging, precision
    std::vector<Job *> jobs;
    RunDesc *d_descs = nullptr;
    double *d_ehist = nullptr;  // [n][SEG][2] (CVD)
    cudaStream_t stream = nullptr;
};

}  // namespace

struct pfc_engine {
    pfc_engine_opts opts{};
    Context *ctx = nullptr;
    cudaStream_t main = nullptr;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;  // guards jobs, queue, events, stop, wake and Job::state / cancel_req
    std::condition_variable cv_sched, cv_events;
    std::map<uint64_t, std::unique_ptr<Job>> jobs;
    std::deque<Job *> queue;  // pending jobs in submission order
    std::deque<pfc_event> events;
    uint64_t next_id = 1;
    bool stop = false;
    bool wake = false;  // something for an idle scheduler to look at

    // scheduler-thread state
    std::vector<Job *> active;
    std::vector<Cohort> cohorts;
    bool composition_changed = true;
    cudaGraphExec_t graph = nullptr;
    double reserved = 0.0;
    DevScratch atoms_scratch, cvd_scratch;
    std::vector<cudaEvent_t> join_events;
    cudaEvent_t fork_event = nullptr;
    double *h_ehist = nullptr;  // pinned staging for CVD energy slots, one area per segment
    size_t h_ehist_len = 0, ehist_slots = 0;

    // writer thread
    std::mutex wmu;
    std::condition_variable wcv;
    std::deque<std::function<void()>> wtasks;
    bool wstop = false;

    std::thread sched_thread, writer_thread;

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

void post(pfc_engine *e, const JobTimes &j, int type, int status, int step, int atoms = 0, double energy = 0.0,
          double mass = 0.0, double t_finish = 0.0) {
    pfc_event ev{};
    ev.job = j.id;
    ev.type = type;
    ev.status = status;
    ev.step = step;
    ev.atoms = atoms;
    ev.energy = energy;
    ev.mass = mass;
    ev.t_submit = j.t_submit;
    ev.t_admit = j.t_admit;
    ev.t_event = e->now();
    ev.t_finish = t_finish;
    std::lock_guard<std::mutex> lk(e->mu);
    e->events.push_back(ev);
    e->cv_events.notify_all();
}

// Queue work for the writer thread (file output, then the events that follow it).
void write_task(pfc_engine *e, std::function<void()> f) {
    std::lock_guard<std::mutex> lk(e->wmu);
    e->wtasks.push_back(std::move(f));
    e->wcv.notify_one();
}

void writer_main(pfc_engine *e) {
    for (;;) {
        std::function<void()> f;
        {
            std::unique_lock<std::mutex> lk(e->wmu);
            e->wcv.wait(lk, [&] { return e->wstop || !e->wtasks.empty(); });
            if (e->wtasks.empty()) return;
            f = std::move(e->wtasks.front());
            e->wtasks.pop_front();
        }
        f();
    }
}

void set_state(pfc_engine *e, Job *j, State s) {
    std::lock_guard<std::mutex> lk(e->mu);
    j->state = s;
    e->wake = true;  // an Elastic job may be waiting for this one
    e->cv_sched.notify_all();
}

// ---------------------------------------------------------------------------
// Cohorts and the captured regular steps
// ---------------------------------------------------------------------------
void free_cohorts(pfc_engine *e) {
    if (e->graph) {
        cudaGraphExecDestroy(e->graph);
        e->graph = nullptr;
    }
    for (auto &c : e->cohorts) {
        if (c.d_descs) cudaFree(c.d_descs);
        if (c.d_ehist) cudaFree(c.d_ehist);
        if (c.stream) cudaStreamDestroy(c.stream);
    }
    e->cohorts.clear();
    for (auto ev : e->join_events) cudaEventDestroy(ev);
    e->join_events.clear();
}

int build_cohorts(pfc_engine *e) {
    free_cohorts(e);
    for (Job *j : e->active) {
        Cohort *c = nullptr;
        for (auto &x : e->cohorts)
            if (x.model == j->spec.kind && x.L == j->L && x.M == j->M && x.CT == j->run->desc.CT &&
                x.stage == j->run->desc.stage && x.prec == j->run->p.precision)
                c = &x;
        if (!c) {
            e->cohorts.push_back(Cohort{});
            c = &e->cohorts.back();
            c->model = j->spec.kind;
            c->L = j->L;
            c->M = j->M;
            c->CT = j->run->desc.CT;
            c->stage = j->run->desc.stage;
            c->prec = j->run->p.precision;
        }
        c->jobs.push_back(j);
    }
    size_t slots = 0;
    for (auto &c : e->cohorts) {
        const int n = (int)c.jobs.size();
        PFC_CUDA_TRY(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        PFC_CUDA_TRY(cudaMalloc(&c.d_descs, n * sizeof(RunDesc)));
        if (c.model == PFC_JOB_CVD) {
            PFC_CUDA_TRY(cudaMalloc(&c.d_ehist, (size_t)n * SEG * 2 * sizeof(double)));
            slots += (size_t)n * SEG * 2;
        }
        std::vector<RunDesc> h(n);
        for (int i = 0; i < n; ++i) {
            h[i] = c.jobs[i]->run->desc;
            h[i].ehist = c.d_ehist ? c.d_ehist + (size_t)i * SEG * 2 : nullptr;
        }
        PFC_CUDA_TRY(cudaMemcpyAsync(c.d_descs, h.data(), n * sizeof(RunDesc), cudaMemcpyHostToDevice, e->main));
        PFC_CUDA_TRY(prepare_size(c.L, c.M, c.CT, c.stage, c.prec));
        cudaEvent_t ev;
        PFC_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        e->join_events.push_back(ev);
    }
    // staging for every segment of a quantum (the regular ones and the final step)
    e->ehist_slots = slots;
    const size_t need = slots * (size_t)(e->opts.quantum_steps / SEG + 2);
    if (need > e->h_ehist_len) {
        if (e->h_ehist) cudaFreeHost(e->h_ehist);
        e->h_ehist = nullptr;
        e->h_ehist_len = 0;
        PFC_CUDA_TRY(cudaMallocHost(&e->h_ehist, need * sizeof(double)));
        e->h_ehist_len = need;
    }
    PFC_CUDA_TRY(cudaStreamSynchronize(e->main));
    e->composition_changed = false;
    return PFC_OK;
}

// One regular step of a cohort: Misfit row + column sweeps; CVD the same with the
// energy analysis that ends every CVD step, its sums going to energy slot `slot`.
// row_done: the step's row work was done by the previous step's analysis; next_row
// (mixed-precision CVD cohorts): the analysis also does the next step's row work (the
// same operations as the row kernel, so the same bits).
int cohort_step(pfc_engine *e, Cohort &c, int slot, cudaStream_t st, bool row_done = false, bool next_row = false) {
    const int n = (int)c.jobs.size();
    const TwiddleSet &tw = e->ctx->tw;
    if (!row_done) PFC_CUDA_TRY(launch_row_step(c.d_descs, n, c.L, c.M, c.prec, tw, st));
    if (c.model == PFC_JOB_MISFIT) {
        PFC_CUDA_TRY(launch_col_step(c.d_descs, n, c.L, c.M, c.CT, c.stage, COL_STEP, c.prec, tw, st));
    } else {
        PFC_CUDA_TRY(launch_col_step(c.d_descs, n, c.L, c.M, c.CT, c.stage, COL_STEP_CHECKPOINT, c.prec, tw, st));
        if (next_row)
            PFC_CUDA_TRY(launch_row_analysis_step_mixed(c.d_descs, n, c.L, c.M, tw, st));
        else
            PFC_CUDA_TRY(launch_row_analysis(c.d_descs, n, c.L, c.M, c.prec, tw, st));
        PFC_CUDA_TRY(launch_reduce_runs(c.d_descs, n, c.jobs[0]->run->nparts, slot, st));  // the runs' shared count
    }
    return PFC_OK;
}

// `len` regular steps of every cohort, each cohort on its own stream (fork / join
// through events, so that the same sequence can be captured into a graph).
int enqueue_steps(pfc_engine *e, int len) {
    PFC_CUDA_TRY(cudaEventRecord(e->fork_event, e->main));
    for (size_t i = 0; i < e->cohorts.size(); ++i) {
        Cohort &c = e->cohorts[i];
        PFC_CUDA_TRY(cudaStreamWaitEvent(c.stream, e->fork_event, 0));
        const bool fuse = c.model == PFC_JOB_CVD && c.prec == PFC_PRECISION_MIXED;
        for (int s = 0; s < len; ++s) {
            const int rc = cohort_step(e, c, s, c.stream, fuse && s > 0, fuse && s + 1 < len);
            if (rc != PFC_OK) return rc;
        }
        PFC_CUDA_TRY(cudaEventRecord(e->join_events[i], c.stream));
        PFC_CUDA_TRY(cudaStreamWaitEvent(e->main, e->join_events[i], 0));
    }
    return PFC_OK;
}

int run_segment(pfc_engine *e, int len) {
    if (len != SEG) return enqueue_steps(e, len);
    if (!e->graph) {
        cudaGraph_t g = nullptr;
        PFC_CUDA_TRY(cudaStreamBeginCapture(e->main, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_steps(e, SEG);
        const cudaError_t ce = cudaStreamEndCapture(e->main, &g);
        if (rc != PFC_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_error(ce, "cudaStreamEndCapture");
        const cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return cuda_error(ie, "cudaGraphInstantiate");
    }
    PFC_CUDA_TRY(cudaGraphLaunch(e->graph, e->main));
    return PFC_OK;
}

// Queue the copy of every CVD cohort's energy slots to the staging area of segment
// `seg`; unpack_energy_slots moves them into each job's per-quantum history after the
// quantum's synchronisation.
int copy_energy_slots(pfc_engine *e, int seg) {
    size_t base = 0;
    for (auto &c : e->cohorts) {
        if (c.model != PFC_JOB_CVD) continue;
        const size_t n = c.jobs.size() * SEG * 2;
        PFC_CUDA_TRY(cudaMemcpyAsync(e->h_ehist + (size_t)seg * e->ehist_slots + base, c.d_ehist, n * sizeof(double),
                                     cudaMemcpyDeviceToHost, e->main));
        base += n;
    }
    return PFC_OK;
}

void unpack_energy_slots(pfc_engine *e, const std::vector<int> &seg_len) {
    int off = 0;
    for (size_t k = 0; k < seg_len.size(); ++k) {
        size_t base = 0;
        for (auto &c : e->cohorts) {
            if (c.model != PFC_JOB_CVD) continue;
            for (size_t i = 0; i < c.jobs.size(); ++i) {
                const double *src = e->h_ehist + k * e->ehist_slots + base + i * SEG * 2;
                Job *j = c.jobs[i];
                for (int s = 0; s < seg_len[k]; ++s) {
                    j->ehist[2 * (off + s)] = src[2 * s];
                    j->ehist[2 * (off + s) + 1] = src[2 * s + 1];
                }
            }
            base += c.jobs.size() * SEG * 2;
        }
        off += seg_len[k];
    }
}

// ---------------------------------------------------------------------------
// Checkpoints and completion
// ---------------------------------------------------------------------------
int copy_fields(pfc_engine *e, Job *j, std::shared_ptr<std::vector<float>> &phi,
                std::shared_ptr<std::vector<float>> &con) {
    const long P = j->run->P;
    phi = std::make_shared<std::vector<float>>(P);
    con = std::make_shared<std::vector<float>>(P);
    PFC_CUDA_TRY(cudaMemcpyAsync(phi->data(), j->run->desc.psi_real, P * sizeof(float), cudaMemcpyDeviceToHost, e->main));
    PFC_CUDA_TRY(cudaMemcpyAsync(con->data(), j->run->desc.con_real, P * sizeof(float), cudaMemcpyDeviceToHost, e->main));
    PFC_SYNC_CHECKED(e->ctx, e->main);
    return PFC_OK;
}

void timestamp_line(const std::string &outdir, int step) {
    std::ofstream log(opath(outdir, "checkpoint_timestamps.txt"), std::ios::out | std::ios::app);
    if (log.is_open()) log << "step " << step << " timestamp_ms " << now_ms() << std::endl;
}

// Misfit checkpoint after the checkpoint-mode step: energy, Phimax, fields (the
// sequence of the CLI's pfc_run_advance(..., 1) + Phimax + checkpoint files).
int misfit_checkpoint(pfc_engine *e, Job *j) {
    pfc_run *r = j->run;
    PFC_CUDA_TRY(launch_row_analysis(r->d_desc, 1, r->L, r->M, r->p.precision, e->ctx->tw, e->main));
    PFC_CUDA_TRY(launch_reduce_fixed(r->desc.partials, r->nparts, 2, 2, r->d_scratch, e->main));
    r->fields_valid = true;
    r->energy_valid = true;
    const long cap = (long)r->L * r->M + 1;
    if (!e->atoms_scratch.ensure(cap * 5 * sizeof(double))) return set_error(PFC_E_NOMEM, "Phimax scratch");
    int count = 0, raw = 0;
    int rc = phimax_misfit_dev(r->desc.psi_real, r->desc.con_real, r->L, r->M, r->p.dx, r->p.con0,
                               (double *)e->atoms_scratch.p, (int)cap, &count, &raw, e->main);
    if (rc != PFC_OK) return rc;
    auto atoms = std::make_shared<std::vector<double>>((size_t)count * 5);
    double sums[2];
    PFC_CUDA_TRY(cudaMemcpyAsync(atoms->data(), e->atoms_scratch.p, atoms->size() * sizeof(double),
                                 cudaMemcpyDeviceToHost, e->main));
    PFC_CUDA_TRY(cudaMemcpyAsync(sums, r->d_scratch, sizeof(sums), cudaMemcpyDeviceToHost, e->main));
    std::shared_ptr<std::vector<float>> phi, con;
    rc = copy_fields(e, j, phi, con);
    if (rc != PFC_OK) return rc;
    const double en = sums[0] / r->L / r->M / r->N, ma = sums[1] / r->L / r->M / r->N;
    const int kd = j->t;
    const int natoms = count_misfit_atoms(*atoms, count);
    j->phi = phi;
    j->con = con;
    const std::string outdir = j->outdir;
    const int L = r->L, M = r->M, N = r->N;
    const JobTimes jt = j->times();
    write_task(e, [e, outdir, kd, atoms, count, phi, con, L, M, N, en, ma, natoms, jt] {
        int status = PFC_OK;
        if (!outdir.empty()) {
            write_phimax_misfit(outdir, kd, *atoms, count);
            if (!write_checkpoint_fields(outdir, kd, phi->data(), con->data(), L, M, N)) status = PFC_E_IO;
            append_energy_line(outdir, kd, en, ma);
            timestamp_line(outdir, kd);
        }
        post(e, jt, PFC_EV_CHECKPOINT, status, kd, natoms, en, ma);
    });
    return PFC_OK;
}

// CVD after a quantum of q steps: the energy lines of its steps; the fields when a
// checkpoint (or the end) was reached.
int cvd_after_quantum(pfc_engine *e, Job *j, int q) {
    pfc_run *r = j->run;
    const int t_end = j->t;
    const int first = t_end - q;  // 0-based loop index of the quantum's first step
    std::vector<std::pair<double, double>> lines(q);
    for (int s = 0; s < q; ++s)
        lines[s] = {j->ehist[2 * s] / r->L / r->M / r->N, j->ehist[2 * s + 1] / r->L / r->M / r->N};
    std::shared_ptr<std::vector<float>> phi, con;
    const bool ckpt = cvd_ckpt(*j, t_end);
    if (ckpt || t_end == j->spec.steps) {
        const int rc = copy_fields(e, j, phi, con);
        if (rc != PFC_OK) return rc;
        j->phi = phi;
        j->con = con;
    }
    // the checkpoint's atom analysis (CVD:427, 1067-1520) on the resident field
    auto ca = std::make_shared<CvdAnalysis>();
    if (ckpt) {
        const int rc = cvd_analyze(r->desc.psi_real, r->L, r->M, r->N, r->p.dx, r->p.u0, t_end - 1, e->main,
                                   e->cvd_scratch, *ca);
        if (rc != PFC_OK) return rc;
    }
    const std::string outdir = j->outdir;
    const int L = r->L, M = r->M, N = r->N;
    const float dx = r->p.dx;
    const JobTimes jt = j->times();
    write_task(e, [e, outdir, first, q, lines, ckpt, phi, con, L, M, N, dx, ca, jt] {
        int status = PFC_OK;
        // energy.txt gets one line per step, kd = the step's 0-based loop index (CVD:442);
        // the checkpoint's files come before its energy line, as in the CLI
        for (int s = 0; s < q; ++s) {
            const int kd = first + s;
            if (outdir.empty()) continue;
            if (ckpt && s == q - 1) {
                write_cvd_files(outdir, L, M, N, dx, *ca);
                if (!write_checkpoint_fields(outdir, kd, phi->data(), con->data(), L, M, N)) status = PFC_E_IO;
                timestamp_line(outdir, kd);
            }
            append_energy_line(outdir, kd, lines[s].first, lines[s].second);
        }
        int natoms = 0;
        for (int i = 0; i < ca->count; ++i) natoms += ca->rec[4 * i] >= 0 ? 1 : 0;
        if (ckpt) post(e, jt, PFC_EV_CHECKPOINT, status, first + q - 1, natoms, lines[q - 1].first, lines[q - 1].second);
    });
    return PFC_OK;
}

void finish_job(pfc_engine *e, Job *j, int type, int status) {
    if (j->run) {
        pfc_run_destroy(j->run);
        j->run = nullptr;
        e->reserved -= j->bytes;
    }
    e->active.erase(std::remove(e->active.begin(), e->active.end(), j), e->active.end());
    e->composition_changed = true;
    const State s = type == PFC_EV_DONE ? State::Done : (type == PFC_EV_CANCELLED ? State::Cancelled : State::Failed);
    const JobTimes jt = j->times();
    const int step = j->t;
    const double t_finish = e->now();
    // the state changes and the event is posted after the job's queued files are written
    write_task(e, [e, j, s, jt, type, status, step, t_finish] {
        set_state(e, j, s);
        post(e, jt, type, status, step, 0, 0.0, 0.0, t_finish);
    });
}

// ---------------------------------------------------------------------------
// Admission
// ---------------------------------------------------------------------------
int admit(pfc_engine *e, Job *j) {
    pfc_run_params p = j->spec.params;
    p.model = j->spec.kind;
    p.device = e->opts.device;
    if (!j->outdir.empty()) {
        std::string why;
        if (!make_dir(j->outdir, &why)) return set_error(PFC_E_IO, "cannot create outdir " + j->outdir + ": " + why);
        write_run_config(j->outdir, p, j->spec.steps, j->spec.mod);
        std::ofstream log(opath(j->outdir, "checkpoint_timestamps.txt"), std::ios::out | std::ios::trunc);
        if (log.is_open()) log << "# Checkpoint timestamps - Step number and milliseconds since epoch" << std::endl;
    }
    pfc_run *r = nullptr;
    int rc = pfc_run_create(&p, &r);
    if (rc != PFC_OK) return rc;
    r->stream = e->main;  // the run's own calls now order after the engine's work
    j->run = r;
    j->L = r->L;
    j->M = r->M;
    j->N = r->N;
    j->t = 0;
    j->t_admit = e->now();
    if (j->spec.kind == PFC_JOB_CVD) j->ehist.assign((size_t)2 * e->opts.quantum_steps, 0.0);
    if (j->spec.kind == PFC_JOB_MISFIT && !j->outdir.empty()) {
        // the initial fields are checkpoint 0 (MIS:464-470)
        std::shared_ptr<std::vector<float>> phi, con;
        rc = copy_fields(e, j, phi, con);
        if (rc != PFC_OK) return rc;
        const std::string outdir = j->outdir;
        const int L = r->L, M = r->M, N = r->N;
        write_task(e, [outdir, phi, con, L, M, N] { write_checkpoint_fields(outdir, 0, phi->data(), con->data(), L, M, N); });
    }
    return PFC_OK;
}

// Elastic job: analyse the source job's final fields or every checkpoint in input_dir.
void run_elastic(pfc_engine *e, Job *j) {
    const float dx = j->spec.params.dx > 0.0f ? j->spec.params.dx : 0.125f;
    const float benchel = j->spec.benchel > 0.0f ? j->spec.benchel : 1.7f;
    std::vector<std::pair<int, std::shared_ptr<std::vector<float>>>> fields;
    int L = 0, M = 0, N = 1;
    int status = PFC_OK;
    j->t_admit = e->now();
    if (j->spec.source_job) {
        std::shared_ptr<std::vector<float>> phi;
        {
            std::lock_guard<std::mutex> lk(e->mu);
            auto it = e->jobs.find(j->spec.source_job);
            if (it != e->jobs.end() && it->second->state == State::Done) {
                phi = it->second->phi;
                L = it->second->L;
                M = it->second->M;
                N = it->second->N;
                fields.push_back({it->second->spec.steps, phi});
            }
        }
        if (!phi) status = set_error(PFC_E_STATE, "source job has no fields");
    } else {
        for (int kd : collect_steps(j->input_dir)) {
            int l = 0, m = 0, n = 0;
            auto f = std::make_shared<std::vector<float>>();
            if (!read_vti(input_file(j->input_dir, "phi_", kd), l, m, n, *f)) {
                status = set_error(PFC_E_IO, "can't open input file: " + input_file(j->input_dir, "phi_", kd));
                break;
            }
            L = l;
            M = m;
            N = n;
            fields.push_back({kd, f});
        }
        if (status == PFC_OK && fields.empty()) status = set_error(PFC_E_IO, "no checkpoints in input_dir");
    }
    if (status == PFC_OK && !j->outdir.empty()) {
        std::string why;
        if (!make_dir(j->outdir, &why)) status = set_error(PFC_E_IO, "cannot create outdir " + j->outdir + ": " + why);
    }
    DevScratch scratch;
    const JobTimes jt = j->times();
    for (auto &kv : fields) {
        if (status != PFC_OK) break;
        auto res = std::make_shared<ElasticResult>();
        status = elastic_analyze(kv.second->data(), L, M, N, dx, benchel, e->main, scratch, *res);
        if (status != PFC_OK) break;
        int total = 0;
        for (int i = 0; i < res->n; ++i) total += res->x[i] >= 0 ? 1 : 0;
        const std::string outdir = j->outdir;
        const int kd = kv.first;
        write_task(e, [e, outdir, kd, res, total, jt] {
            if (!outdir.empty()) {
                std::ostringstream diag;  // the CLI prints this line to stderr; the engine drops it
                write_elastic_files(outdir, kd, *res, diag);
            }
            post(e, jt, PFC_EV_CHECKPOINT, PFC_OK, kd, total);
        });
        j->t = kd;
    }
    finish_job(e, j, status == PFC_OK ? PFC_EV_DONE : PFC_EV_FAILED, status);
}

// ---------------------------------------------------------------------------
// Scheduler
// ---------------------------------------------------------------------------
int quantum(pfc_engine *e) {
    int q = e->opts.quantum_steps;
    for (Job *j : e->active) q = std::min(q, steps_to_event(*j));
    if (q <= 0) return PFC_OK;
    if (e->composition_changed) {
        const int rc = build_cohorts(e);
        if (rc != PFC_OK) return rc;
    }
    // Misfit runs that checkpoint at the end of this quantum take their last step in
    // checkpoint mode; everything else runs as regular steps.
    std::vector<Job *> ckpt;
    for (Job *j : e->active)
        if (j->spec.kind == PFC_JOB_MISFIT && misfit_ckpt(*j, j->t + q)) ckpt.push_back(j);
    const int regular = ckpt.empty() ? q : q - 1;
    std::vector<int> seg_len;
    for (int done = 0; done < regular;) {
        const int len = std::min(SEG, regular - done);
        int rc = run_segment(e, len);
        if (rc == PFC_OK) rc = copy_energy_slots(e, (int)seg_len.size());
        if (rc != PFC_OK) return rc;
        seg_len.push_back(len);
        done += len;
    }
    if (!ckpt.empty()) {
        // final step: every cohort's row sweep, then the column sweep per run with its mode
        const TwiddleSet &tw = e->ctx->tw;
        for (auto &c : e->cohorts) {
            if (c.model == PFC_JOB_CVD) {
                const int rc = cohort_step(e, c, 0, e->main);
                if (rc != PFC_OK) return rc;
                continue;
            }
            PFC_CUDA_TRY(launch_row_step(c.d_descs, (int)c.jobs.size(), c.L, c.M, c.prec, tw, e->main));
            for (Job *j : c.jobs) {
                const bool ck = std::find(ckpt.begin(), ckpt.end(), j) != ckpt.end();
                PFC_CUDA_TRY(launch_col_step(j->run->d_desc, 1, c.L, c.M, c.CT, c.stage,
                                             ck ? COL_STEP_CHECKPOINT : COL_STEP, c.prec, tw, e->main));
            }
        }
        const int rc = copy_energy_slots(e, (int)seg_len.size());
        if (rc != PFC_OK) return rc;
        seg_len.push_back(1);
    }
    PFC_SYNC_CHECKED(e->ctx, e->main);
    unpack_energy_slots(e, seg_len);
    for (Job *j : e->active) {
        j->t += q;
        j->run->t = j->t;
        j->run->fields_valid = j->spec.kind == PFC_JOB_CVD;
        j->run->energy_valid = false;
    }
    // a run whose fields went non-finite in this quantum fails alone; the others go on
    // (their kernels never read another run's data)
    for (Job *j : std::vector<Job *>(e->active)) {
        if (*j->run->h_nonfinite == 0) continue;
        ckpt.erase(std::remove(ckpt.begin(), ckpt.end(), j), ckpt.end());
        finish_job(e, j, PFC_EV_FAILED, PFC_E_NONFINITE);
    }
    for (Job *j : ckpt) {
        const int rc = misfit_checkpoint(e, j);
        if (rc != PFC_OK) return rc;
    }
    for (Job *j : std::vector<Job *>(e->active)) {
        if (j->spec.kind == PFC_JOB_CVD) {
            const int rc = cvd_after_quantum(e, j, q);
            if (rc != PFC_OK) return rc;
        }
        if (j->t >= j->spec.steps) finish_job(e, j, PFC_EV_DONE, PFC_OK);
    }
    return PFC_OK;
}

void scheduler_main(pfc_engine *e) {
    cudaSetDevice(e->opts.device);
    for (;;) {
        std::vector<Job *> admit_now, elastic_now, cancel_now;
        bool stopping = false;
        {
            std::unique_lock<std::mutex> lk(e->mu);
            if (e->active.empty() && !e->stop)
                e->cv_sched.wait_for(lk, std::chrono::milliseconds(50), [&] { return e->stop || e->wake; });
            e->wake = false;
            stopping = e->stop;
            for (Job *j : e->active)
                if (j->cancel_req || stopping) cancel_now.push_back(j);
            // queued jobs in order: cancelled ones leave, Elastic jobs whose input is ready
            // run, simulations are admitted while they fit (the first that does not fit
            // holds the ones behind it)
            double reserved = e->reserved;
            int nactive = (int)e->active.size();
            bool blocked = false;
            for (auto it = e->queue.begin(); it != e->queue.end();) {
                Job *j = *it;
                if (j->cancel_req || stopping) {
                    cancel_now.push_back(j);
                    it = e->queue.erase(it);
                    continue;
                }
                if (j->spec.kind == PFC_JOB_ELASTIC) {
                    bool ready = !j->spec.source_job;
                    if (!ready) {
                        auto src = e->jobs.find(j->spec.source_job);
                        ready = src == e->jobs.end() || src->second->state == State::Done ||
                                src->second->state == State::Failed || src->second->state == State::Cancelled;
                    }
                    if (ready) {
                        elastic_now.push_back(j);
                        it = e->queue.erase(it);
                    } else {
                        ++it;
                    }
                    continue;
                }
                const bool fits = reserved + j->bytes <= e->opts.hbm_budget_bytes &&
                                  (e->opts.max_active <= 0 || nactive < e->opts.max_active);
                if (!blocked && fits) {
                    reserved += j->bytes;
                    ++nactive;
                    admit_now.push_back(j);
                    it = e->queue.erase(it);
                } else {
                    blocked = true;
                    ++it;
                }
            }
        }
        for (Job *j : cancel_now) {
            if (j->run) {
                finish_job(e, j, PFC_EV_CANCELLED, PFC_OK);
            } else {
                const JobTimes jt = j->times();
                const double t_finish = e->now();
                write_task(e, [e, j, jt, t_finish] {
                    set_state(e, j, State::Cancelled);
                    post(e, jt, PFC_EV_CANCELLED, PFC_OK, 0, 0, 0.0, 0.0, t_finish);
                });
            }
        }
        if (stopping) {
            free_cohorts(e);
            return;
        }
        for (Job *j : admit_now) {
            const int rc = admit(e, j);
            if (rc != PFC_OK) {
                if (j->run) pfc_run_destroy(j->run);
                j->run = nullptr;
                const JobTimes jt = j->times();
                const double t_finish = e->now();
                write_task(e, [e, j, jt, rc, t_finish] {
                    set_state(e, j, State::Failed);
                    post(e, jt, PFC_EV_FAILED, rc, 0, 0, 0.0, 0.0, t_finish);
                });
                continue;
            }
            e->reserved += j->bytes;
            e->active.push_back(j);
            e->composition_changed = true;
            set_state(e, j, State::Active);
            post(e, j->times(), PFC_EV_ADMITTED, PFC_OK, 0);
        }
        for (Job *j : elastic_now) {
            set_state(e, j, State::Active);
            run_elastic(e, j);
        }
        if (!e->active.empty()) {
            const int rc = quantum(e);
            if (rc != PFC_OK) {
                cudaStreamSynchronize(e->main);
                for (Job *j : std::vector<Job *>(e->active)) finish_job(e, j, PFC_EV_FAILED, rc);
            }
        }
    }
}

int take_events(pfc_engine *e, pfc_event *ev, int max, int *n) {
    int k = 0;
    while (k < max && !e->events.empty()) {
        ev[k++] = e->events.front();
        e->events.pop_front();
    }
    *n = k;
    return PFC_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" int pfc_engine_create(const pfc_engine_opts *opts, pfc_engine **out) {
    if (!out) return set_error(PFC_E_INVALID, "null output pointer");
    *out = nullptr;
    pfc_engine_opts o{};
    if (opts) o = *opts;
    if (o.quantum_steps <= 0) o.quantum_steps = 64;
    Context *ctx = nullptr;
    int rc = get_context(o.device, &ctx);
    if (rc != PFC_OK) return rc;
    PFC_CUDA_TRY(cudaSetDevice(o.device));
    size_t free_b = 0, total_b = 0;
    PFC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const double cap = (double)free_b - 2e9;  // headroom for analysis scratch and the runtime
    if (o.hbm_budget_bytes <= 0.0) o.hbm_budget_bytes = 150e9;
    if (o.hbm_budget_bytes > cap) o.hbm_budget_bytes = cap;
    if (o.hbm_budget_bytes <= 0.0) return set_error(PFC_E_NOMEM, "no device memory for the engine");
    auto *e = new pfc_engine();
    e->opts = o;
    e->ctx = ctx;
    e->t0 = std::chrono::steady_clock::now();
    cudaError_t ce = cudaStreamCreateWithFlags(&e->main, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&e->fork_event, cudaEventDisableTiming);
    if (ce != cudaSuccess) {
        if (e->main) cudaStreamDestroy(e->main);
        delete e;
        return cuda_error(ce, "engine stream");
    }
    e->writer_thread = std::thread(writer_main, e);
    e->sched_thread = std::thread(scheduler_main, e);
    *out = e;
    return PFC_OK;
}

extern "C" int pfc_engine_destroy(pfc_engine *e) {
    if (!e) return PFC_OK;
    {
        std::lock_guard<std::mutex> lk(e->mu);
        e->stop = true;
        e->cv_sched.notify_all();
    }
    e->sched_thread.join();
    {
        std::lock_guard<std::mutex> lk(e->wmu);
        e->wstop = true;
        e->wcv.notify_all();
    }
    e->writer_thread.join();
    cudaSetDevice(e->opts.device);
    free_cohorts(e);
    if (e->h_ehist) cudaFreeHost(e->h_ehist);
    if (e->fork_event) cudaEventDestroy(e->fork_event);
    if (e->main) cudaStreamDestroy(e->main);
    delete e;
    return PFC_OK;
}

// A job from its spec, checked; the caller queues it.
static int make_job(pfc_engine *e, const pfc_job *job, std::unique_ptr<Job> &out) {
    auto j = std::make_unique<Job>();
    j->spec = *job;
    j->outdir = job->outdir ? job->outdir : "";
    j->input_dir = job->input_dir ? job->input_dir : "";
    j->spec.outdir = nullptr;
    j->spec.input_dir = nullptr;
    if (job->kind == PFC_JOB_MISFIT || job->kind == PFC_JOB_CVD) {
        pfc_run_params p = job->params;
        p.model = job->kind;
        if (!fused_path(p.precision))
            return set_error(PFC_E_INVALID, "engine runs use the fused paths (mixed or FP32 precision)");
        if (p.N != 1) return set_error(PFC_E_INVALID, "engine runs are 2-D (N = 1)");
        if (job->steps <= 0 || job->mod <= 0) return set_error(PFC_E_INVALID, "steps and mod must be > 0");
        double b = 0.0;
        const int rc = pfc_run_bytes(&p, &b);
        if (rc != PFC_OK) return rc;
        j->bytes = b;
        if (b > e->opts.hbm_budget_bytes) return set_error(PFC_E_NOMEM, "run larger than the engine's memory budget");
    } else if (job->kind == PFC_JOB_ELASTIC) {
        if (!job->source_job && j->input_dir.empty())
            return set_error(PFC_E_INVALID, "elastic job needs source_job or input_dir");
    } else {
        return set_error(PFC_E_INVALID, "unknown job kind");
    }
    out = std::move(j);
    return PFC_OK;
}

// An Elastic job's source must be a Misfit or CVD job of this engine (e->mu held);
// `pending` are jobs queued in the same call, ahead of this one.
static bool source_ok(pfc_engine *e, const pfc_job *job, const std::vector<std::unique_ptr<Job>> &pending,
                      uint64_t first_id) {
    if (job->kind != PFC_JOB_ELASTIC || !job->source_job) return true;
    auto it = e->jobs.find(job->source_job);
    if (it != e->jobs.end()) return it->second->spec.kind != PFC_JOB_ELASTIC;
    const uint64_t k = job->source_job - first_id;
    return job->source_job >= first_id && k < pending.size() && pending[k] && pending[k]->spec.kind != PFC_JOB_ELASTIC;
}

extern "C" int pfc_submit(pfc_engine *e, const pfc_job *job, uint64_t *id) {
    if (!job) return set_error(PFC_E_INVALID, "null argument");
    return pfc_submit_many(e, job, 1, id);
}

extern "C" int pfc_submit_many(pfc_engine *e, const pfc_job *jobs, int n, uint64_t *ids) {
    if (!e || !jobs || !ids || n <= 0) return set_error(PFC_E_INVALID, "null argument or empty job list");
    std::vector<std::unique_ptr<Job>> js(n);
    for (int i = 0; i < n; ++i) {
        const int rc = make_job(e, &jobs[i], js[i]);
        if (rc != PFC_OK) return n > 1 ? set_error(rc, "job " + std::to_string(i) + ": " + pfc_last_error()) : rc;
    }
    std::lock_guard<std::mutex> lk(e->mu);
    const uint64_t first = e->next_id;
    for (int i = 0; i < n; ++i)
        if (!source_ok(e, &jobs[i], js, first))
            return set_error(PFC_E_INVALID, (n > 1 ? "job " + std::to_string(i) + ": " : std::string()) +
                                                "source_job is not a Misfit or CVD job of this engine");
    const double t = e->now();
    for (int i = 0; i < n; ++i) {
        Job *j = js[i].get();
        j->id = e->next_id++;
        j->t_submit = t;
        ids[i] = j->id;
        e->queue.push_back(j);
        e->jobs[j->id] = std::move(js[i]);
    }
    e->wake = true;
    e->cv_sched.notify_all();
    return PFC_OK;
}

extern "C" int pfc_poll(pfc_engine *e, pfc_event *ev, int max, int *n) {
    if (!e || !n || (max > 0 && !ev)) return set_error(PFC_E_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(e->mu);
    return take_events(e, ev, max, n);
}

extern "C" int pfc_wait(pfc_engine *e, pfc_event *ev, int max, int *n, int timeout_ms) {
    if (!e || !n || (max > 0 && !ev)) return set_error(PFC_E_INVALID, "null argument");
    std::unique_lock<std::mutex> lk(e->mu);
    auto ready = [&] { return !e->events.empty(); };
    if (timeout_ms < 0) e->cv_events.wait(lk, ready);
    else e->cv_events.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    return take_events(e, ev, max, n);
}

extern "C" int pfc_cancel(pfc_engine *e, uint64_t id) {
    if (!e) return set_error(PFC_E_INVALID, "null engine");
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(id);
    if (it == e->jobs.end()) return set_error(PFC_E_INVALID, "unknown job");
    Job *j = it->second.get();
    if (j->state == State::Done || j->state == State::Failed || j->state == State::Cancelled)
        return set_error(PFC_E_STATE, "job already finished");
    j->cancel_req = true;
    e->wake = true;
    e->cv_sched.notify_all();
    return PFC_OK;
}

extern "C" int pfc_job_fields(pfc_engine *e, uint64_t id, float *phi, float *con) {
    if (!e) return set_error(PFC_E_INVALID, "null engine");
    std::shared_ptr<std::vector<float>> a, b;
    {
        std::lock_guard<std::mutex> lk(e->mu);
        auto it = e->jobs.find(id);
        if (it == e->jobs.end()) return set_error(PFC_E_INVALID, "unknown job");
        if (it->second->state != State::Done) return set_error(PFC_E_STATE, "job is not done");
        a = it->second->phi;
        b = it->second->con;
    }
    if (!a || !b) return set_error(PFC_E_STATE, "job has no fields");
    if (phi) std::copy(a->begin(), a->end(), phi);
    if (con) std::copy(b->begin(), b->end(), con);
    return PFC_OK;
}

extern "C" int pfc_release(pfc_engine *e, uint64_t id) {
    if (!e) return set_error(PFC_E_INVALID, "null engine");
    std::lock_guard<std::mutex> lk(e->mu);
    auto it = e->jobs.find(id);
    if (it == e->jobs.end()) return set_error(PFC_E_INVALID, "unknown job");
    const State s = it->second->state;
    if (s != State::Done && s != State::Failed && s != State::Cancelled)
        return set_error(PFC_E_STATE, "job is not finished");
    it->second->phi.reset();
    it->second->con.reset();
    return PFC_OK;
}

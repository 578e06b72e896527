// cli.cpp -- pfc_run_cli: the pfc-exp-cli process interface on the GPU engine.
//
// Restates the reference's command-line surface (paths within zhiqing0205/PFC-Exp-GUI):
//   src/experiment/main_cli.cpp:14-88        --model dispatch and global help
//   src/experiment/misfit_uniform_time_seed_fftw_early.cpp:17-309, 311-531
//                                            Misfit options, run_config.txt, time loop,
//                                            checkpoints (Phimax, VTI, energy, timestamps)
//   src/experiment/cvd.cpp:111-203, 215-454  CVD options and time loop
//   src/experiment/elastic.cpp:30-74, 137-289, 304-521
//                                            Elastic options, checkpoint discovery, analysis
//   src/experiment/pfc_common.h:186-269      strict numeric parsers, --outdir creation
// Files are byte-compatible with the reference writers (VTI/PVTI at
// misfit_uniform_time_seed_fftw_early.cpp:1588-1810, text files with std::fixed and
// precision(4)).  Additive options: --grid LxMxN (runtime grid; default 256x256x1)
// and --precision mixed|fp32|fp64|fp64-pure (default mixed: FP32 arrays, FP64
// arithmetic, on every 2-D grid and on 3-D grids with N >= 8; fp64 elsewhere).  Output
// paths are prefixed with --outdir
// instead of changing the process working directory.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <iterator>
#include <limits>
#include <set>
#include <string>
#include <string_view>
#include <vector>

#include "pfc_b200.h"
#include "checkpoint.h"
#include "pfc_engine.h"
#include "sweep.h"

namespace pfc {
int phimax_misfit_dev(const float *d_phi, const float *d_con, int L, int M, float dx, float con0, double *d_out,
                      int cap, int *count, int *raw_count, cudaStream_t st);
int phimax_elastic_dev(const float *d_phi, int L, int M, int N, float dx, double *d_out, int cap, int *count,
                       cudaStream_t st);
int elastic3d_dev(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                  float benchel, double *strain, uint32_t *nb, cudaStream_t st);
int cryst_order_dev(const double *x, const double *y, const double *z, int n, int L, int M, int N, float dx,
                    double *q4, double *q6, cudaStream_t st);
}  // namespace pfc

using namespace pfc;
using namespace pfc::ckpt;
using std::cerr;
using std::cout;
using std::endl;

namespace {

// ---------------------------------------------------------------------------
// Strict parsers (pfc_common.h:186-220)
// ---------------------------------------------------------------------------
bool parse_int(const char *v, int &out) {
    if (!v) return false;
    char *end = nullptr;
    errno = 0;
    long x = strtol(v, &end, 10);
    if (errno != 0 || end == v || *end != '\0') return false;
    if (x < std::numeric_limits<int>::min() || x > std::numeric_limits<int>::max()) return false;
    out = (int)x;
    return true;
}
bool parse_float(const char *v, float &out) {
    if (!v) return false;
    char *end = nullptr;
    errno = 0;
    float x = strtof(v, &end);
    if (errno != 0 || end == v || *end != '\0') return false;
    out = x;
    return true;
}
bool parse_uint(const char *v, unsigned int &out) {
    if (!v) return false;
    char *end = nullptr;
    errno = 0;
    unsigned long long x = strtoull(v, &end, 10);
    if (errno != 0 || end == v || *end != '\0') return false;
    if (x > std::numeric_limits<unsigned int>::max()) return false;
    out = (unsigned int)x;
    return true;
}
bool has_prefix(std::string_view s, std::string_view p) { return s.size() >= p.size() && s.substr(0, p.size()) == p; }

bool parse_grid(const char *v, int &L, int &M, int &N) {
    if (!v) return false;
    int a = 0, b = 0, c = 0;
    char x1 = 0, x2 = 0, extra = 0;
    if (sscanf(v, "%d%c%d%c%d%c", &a, &x1, &b, &x2, &c, &extra) != 5) return false;
    if ((x1 != 'x' && x1 != 'X') || (x2 != 'x' && x2 != 'X')) return false;
    if (a <= 0 || b <= 0 || c <= 0) return false;
    L = a;
    M = b;
    N = c;
    return true;
}
// Without --precision: the mixed path wherever its kernels take the grid (2-D grids, and
// 3-D grids with N >= 8 whose m-pass tile fits), else the plain FP64 path.
int default_precision(pfc_run_params p) {
    p.precision = PFC_PRECISION_MIXED;
    double b = 0.0;
    return pfc_run_bytes(&p, &b) == PFC_OK ? PFC_PRECISION_MIXED : PFC_PRECISION_FP64;
}

bool parse_precision(const char *v, int &out) {
    if (!v) return false;
    std::string s(v);
    if (s == "mixed") out = PFC_PRECISION_MIXED;
    else if (s == "fp32") out = PFC_PRECISION_FP32;
    else if (s == "fp64") out = PFC_PRECISION_FP64;
    else if (s == "fp64-pure") out = PFC_PRECISION_FP64_PURE;
    else return false;
    return true;
}

// --outdir handling (pfc_common.h:249-269): create the directory; files are written
// below it.
bool setup_outdir(const std::string &dir) {
    if (dir.empty()) return true;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) {
        cerr << "Failed to create --outdir '" << dir << "': " << ec.message() << endl;
        return false;
    }
    if (!std::filesystem::is_directory(dir, ec)) {
        cerr << "Failed to chdir to --outdir '" << dir << "': Not a directory" << endl;
        return false;
    }
    return true;
}
struct RunGuard {
    pfc_run *r = nullptr;
    ~RunGuard() {
        if (r) pfc_run_destroy(r);
    }
};

int gpu_fail(const char *what) {
    cerr << "pfc-exp-cli: " << what << ": " << pfc_last_error() << endl;
    return 2;
}

// Shared options of the simulation models.
struct SimOpts {
    float u0, con0, sig, dt, dx, axx;
    int steps, mod;
    unsigned int seed;
    int grainx, grainy, grainz;
    int L = 256, M = 256, N = 1;
    int precision = -1;  // -1: default_precision (mixed where its kernels take the grid)
    int resume = -1;  // --resume <kd>: continue from the run's own checkpoint kd
    std::string outdir;
};

// --resume <kd> (additive option): the state of checkpoint kd is read back from
// phi_<kd>_0.vti / con_<kd>_0.vti in --outdir (the reference's own reader,
// READPHIVTIN / READPHIVTIC at MIS:3019-3190, reads a fixed step only), and the run
// continues with t_state steps taken.  The FP32 state is rebuilt from the Float32
// files, so the continuation equals an uninterrupted run to within rounding; the
// noise stream, counted by step, continues exactly.
int resume_run(pfc_run *r, const SimOpts &o, int kd, int t_state) {
    std::vector<float> f[2];
    const char *pre[2] = {"phi_", "con_"};
    for (int k = 0; k < 2; ++k) {
        int l = 0, m = 0, n = 0;
        const std::string path = opath(o.outdir, input_file("", pre[k], kd));
        if (!read_vti(path, l, m, n, f[k])) {
            cerr << "can't open input file: " << path << endl;
            return 2;
        }
        if (l != o.L || m != o.M || n != o.N) {
            cerr << "pfc-exp-cli: " << path << " holds a " << l << "x" << m << "x" << n << " grid, not " << o.L << "x"
                 << o.M << "x" << o.N << endl;
            return 2;
        }
    }
    std::vector<double> phi(f[0].begin(), f[0].end()), con(f[1].begin(), f[1].end());
    r->t = t_state;
    if (pfc_run_set_fields(r, phi.data(), con.data()) != PFC_OK) return gpu_fail("resume");
    return 0;
}

// ---------------------------------------------------------------------------
// Misfit (MIS:17-309, 311-531)
// ---------------------------------------------------------------------------
void misfit_usage(const char *argv0) {
    cerr << "Usage: " << (argv0 ? argv0 : "pfc-exp-cli") << " --model misfit [options]\n"
         << "Options:\n"
         << "  --u0 <float>        Density/phi mean (default: 0.05)\n"
         << "  --con0 <float>      Concentration mean (default: 0.2)\n"
         << "  --sig <float>       Kernel decay sigma (default: 0.05)\n"
         << "  --dt <float>        Time step (default: 0.05)\n"
         << "  --dx <float>        Space step (default: 0.125)\n"
         << "  --steps <int>       Total iterations (default: 200)\n"
         << "  --mod <int>         Output/analysis interval (default: 25)\n"
         << "  --seed <uint>       Random seed base (default: 20200604)\n"
         << "  --grainx <int>      Initial grains in x (default: 16)\n"
         << "  --grainy <int>      Initial grains in y (default: 16)\n"
         << "  --grainz <int>      Initial grains in z (default: 1)\n"
         << "  --axx <float>       Noise base intensity (default: 0)\n"
         << "  --outdir <path>     Output directory (default: current dir)\n"
         << "  --grid <LxMxN>      Grid (default: 256x256x1)\n"
         << "  --precision <p>     mixed, fp32, fp64 or fp64-pure (default: mixed; fp64 on 3-D grids it does not take)\n"
         << "  --resume <kd>       Continue from checkpoint kd in --outdir\n"
         << "  -h, --help          Show this help\n";
}

// Misfit checkpoint analysis: Phimax_<kd>.txt (MIS:3261-3556) with its stdout lines.
int misfit_phimax(pfc_run *r, const SimOpts &o, const std::vector<float> &phi, const std::vector<float> &con, int kd,
                  DevScratch &scratch) {
    const int L = r->L, M = r->M;
    cout << "o" << "myid=" << 0 << endl;
    cout << "first" << "myid=" << 0 << endl;
    const long cap = (long)L * M + 1;
    if (!scratch.ensure(cap * 5 * sizeof(double))) return gpu_fail("device allocation for Phimax");
    int count = 0, raw = 0;
    if (phimax_misfit_dev(r->desc.psi_real, r->desc.con_real, L, M, o.dx, o.con0, (double *)scratch.p, (int)cap, &count,
                          &raw, r->stream) != PFC_OK)
        return gpu_fail("Phimax");
    std::vector<double> atoms((size_t)count * 5);
    if (cudaMemcpyAsync(atoms.data(), scratch.p, atoms.size() * sizeof(double), cudaMemcpyDeviceToHost, r->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(r->stream) != cudaSuccess)
        return gpu_fail("Phimax copy");
    // debug statistics of the reference (MIS:3310-3330) from the host copy
    double gmin = std::numeric_limits<double>::infinity(), gmax = -std::numeric_limits<double>::infinity();
    int finite_phi = 0, above_cut = 0;
    for (long i = 0; i < (long)L * M; ++i) {
        const double v = phi[i];
        if (!std::isfinite(v)) continue;
        finite_phi++;
        gmin = std::min(gmin, v);
        gmax = std::max(gmax, v);
        if (v > -0.07) above_cut++;
    }
    if (raw == 0) cout << "WARNING: no local maxima found; writing global max fallback point" << endl;
    cout << count << " " << 0 << endl;
    cout << "second" << "myid=" << 0 << endl;
    cout << "third" << "myid=" << 0 << endl;
    const int total = count_misfit_atoms(atoms, count);
    cout << "num_atoms_total=" << total << endl;
    if (total <= 2)
        cout << "phimax_atmposi debug: finite_phi=" << finite_phi << " above_cut=" << above_cut << " phi_min=" << gmin
             << " phi_max=" << gmax << endl;
    write_phimax_misfit(o.outdir, kd, atoms, count);
    (void)con;
    return 0;
}

int append_energy(pfc_run *r, const SimOpts &o, int kd) {
    double e = 0.0, d = 0.0;
    if (pfc_run_energy(r, &e, &d) != PFC_OK) return gpu_fail("energy");
    append_energy_line(o.outdir, kd, e, d);
    return 0;
}

int run_misfit_cli(int argc, char **argv) {
    SimOpts o;
    o.u0 = 0.05f;
    o.con0 = 0.2f;
    o.sig = 0.05f;
    o.dt = 0.05f;
    o.dx = 0.125f;
    o.axx = 0.0f;
    o.steps = 200;
    o.mod = 25;
    o.seed = 20200604u;
    o.grainx = 16;
    o.grainy = 16;
    o.grainz = 1;
    for (int i = 1; i < argc; ++i) {
        if (!argv[i]) continue;
        if (strcmp(argv[i], "-h") == 0 || strcmp(argv[i], "--help") == 0) {
            misfit_usage(argv[0]);
            return 0;
        }
    }
    bool bad = false;
    for (int i = 1; i < argc && !bad; ++i) {
        const char *raw = argv[i];
        if (!raw) continue;
        std::string_view arg(raw);
        auto value = [&](const char *opt) -> const char * {
            const std::string eq = std::string(opt) + "=";
            if (arg == opt) {
                if (i + 1 >= argc) {
                    cerr << "Missing value after " << opt << "\n";
                    return nullptr;
                }
                return argv[++i];
            }
            return raw + eq.size();
        };
        auto is = [&](const char *opt) { return arg == opt || has_prefix(arg, std::string(opt) + "="); };
        if (is("--u0")) bad = !parse_float(value("--u0"), o.u0);
        else if (is("--con0")) bad = !parse_float(value("--con0"), o.con0);
        else if (is("--sig")) bad = !parse_float(value("--sig"), o.sig);
        else if (is("--dt")) bad = !parse_float(value("--dt"), o.dt);
        else if (is("--dx")) bad = !parse_float(value("--dx"), o.dx);
        else if (is("--steps")) bad = !parse_int(value("--steps"), o.steps);
        else if (is("--mod")) bad = !parse_int(value("--mod"), o.mod);
        else if (is("--seed")) bad = !parse_uint(value("--seed"), o.seed);
        else if (is("--grainx")) bad = !parse_int(value("--grainx"), o.grainx);
        else if (is("--grainy")) bad = !parse_int(value("--grainy"), o.grainy);
        else if (is("--grainz")) bad = !parse_int(value("--grainz"), o.grainz);
        else if (is("--axx")) bad = !parse_float(value("--axx"), o.axx);
        else if (is("--grid")) bad = !parse_grid(value("--grid"), o.L, o.M, o.N);
        else if (is("--precision")) bad = !parse_precision(value("--precision"), o.precision);
        else if (is("--resume")) bad = !parse_int(value("--resume"), o.resume) || o.resume < 0;
        else if (is("--outdir")) {
            const char *v = value("--outdir");
            if (!v || *v == '\0') bad = true;
            else o.outdir = v;
        } else {
            cerr << "Unknown option: " << arg << "\n";
            bad = true;
        }
    }
    const int L = o.L, M = o.M, N = o.N;
    if (!bad) {
        if (o.steps <= 0) {
            cerr << "--steps must be > 0\n";
            bad = true;
        } else if (o.dt <= 0.0f) {
            cerr << "--dt must be > 0\n";
            bad = true;
        } else if (o.dx <= 0.0f) {
            cerr << "--dx must be > 0\n";
            bad = true;
        } else if (o.mod <= 0) {
            cerr << "--mod must be > 0\n";
            bad = true;
        } else if (o.grainx <= 0 || o.grainy <= 0 || o.grainz <= 0) {
            cerr << "--grainx/--grainy/--grainz must be > 0\n";
            bad = true;
        } else if (o.grainx > L || o.grainy > M || o.grainz > N) {
            cerr << "--grainx/--grainy/--grainz must not exceed grid dimensions (L=" << L << " M=" << M << " N=" << N
                 << ")\n";
            bad = true;
        }
    }
    if (bad) {
        misfit_usage(argv[0]);
        return 2;
    }
    const float b0 = (o.dx > 0.0f && o.dt > 0.0f && o.axx >= 0.0f) ? (float)sqrt(o.axx / o.dx / o.dx / o.dx / o.dt) : 0.0f;
    if (!setup_outdir(o.outdir)) return 2;
    cerr << "Run config: "
         << "u0=" << o.u0 << " con0=" << o.con0 << " sig=" << o.sig << " dt=" << o.dt << " dx=" << o.dx
         << " steps=" << o.steps << " mod=" << o.mod << " seed=" << o.seed << " grid=(" << L << "," << M << "," << N
         << ")"
         << " grain=(" << o.grainx << "," << o.grainy << "," << o.grainz << ")"
         << " axx=" << o.axx << " b0=" << b0 << " outdir=" << (o.outdir.empty() ? "." : o.outdir) << endl;
    {
        std::ofstream c(opath(o.outdir, "run_config.txt"), std::ios::out | std::ios::trunc);
        if (c.is_open()) {
            c << "model misfit\n";
            c << "u0 " << o.u0 << "\n";
            c << "con0 " << o.con0 << "\n";
            c << "sig " << o.sig << "\n";
            c << "dt " << o.dt << "\n";
            c << "dx " << o.dx << "\n";
            c << "steps " << o.steps << "\n";
            c << "mod " << o.mod << "\n";
            c << "seed " << o.seed << "\n";
            c << "L " << L << "\n";
            c << "M " << M << "\n";
            c << "N " << N << "\n";
            c << "grainx " << o.grainx << "\n";
            c << "grainy " << o.grainy << "\n";
            c << "grainz " << o.grainz << "\n";
            c << "axx " << o.axx << "\n";
            c << "b0 " << b0 << "\n";
        }
    }
    std::ofstream log(opath(o.outdir, "checkpoint_timestamps.txt"),
                      std::ios::out | (o.resume >= 0 ? std::ios::app : std::ios::trunc));
    if (log.is_open()) {
        if (o.resume < 0) log << "# Checkpoint timestamps - Step number and milliseconds since epoch" << endl;
    } else {
        cerr << "Warning: Failed to open checkpoint_timestamps.txt for writing" << endl;
    }

    pfc_run_params p;
    pfc_default_params(PFC_MODEL_MISFIT, &p);
    p.L = L;
    p.M = M;
    p.N = N;
    p.u0 = o.u0;
    p.con0 = o.con0;
    p.sig = o.sig;
    p.dt = o.dt;
    p.dx = o.dx;
    p.axx = o.axx;
    p.grainx = o.grainx;
    p.grainy = o.grainy;
    p.grainz = o.grainz;
    p.seed = o.seed;
    p.precision = o.precision >= 0 ? o.precision : default_precision(p);
    RunGuard g;
    if (pfc_run_create(&p, &g.r) != PFC_OK) return gpu_fail("run setup");
    pfc_run *r = g.r;
    const long P = (long)L * M * N;
    std::vector<float> phi(P), con(P);
    if (o.resume >= 0) {
        const int rc = resume_run(r, o, o.resume, o.resume);
        if (rc != 0) return rc;
    } else {
        if (pfc_run_get_fields_f32(r, phi.data(), con.data()) != PFC_OK) return gpu_fail("initial fields");
        if (!write_checkpoint_fields(o.outdir, 0, phi.data(), con.data(), L, M, N)) {
            cerr << "pfc-exp-cli: failed to write checkpoint files" << endl;
            return 2;
        }
    }
    DevScratch scratch;
    const int progress_every = std::max(1, o.steps / 200);
    int t = o.resume >= 0 ? o.resume : 0;
    while (t < o.steps) {
        // next step at which something is printed or written
        int next = t + 1;
        for (int s = t + 1; s <= o.steps; ++s) {
            if (s == 1 || s % progress_every == 0 || s == o.steps || s % o.mod == 0) {
                next = s;
                break;
            }
        }
        const bool ckpt = (next % o.mod) == 0 || next == o.steps;
        if (pfc_run_advance(r, next - t, ckpt ? 1 : 0) != PFC_OK) return gpu_fail("time step");
        t = next;
        if (t == 1 || t % progress_every == 0 || t == o.steps) {
            if (cudaStreamSynchronize(r->stream) != cudaSuccess) return gpu_fail("time step");
            cout << "PFC_PROGRESS step=" << t << " total=" << o.steps << endl;
        }
        if (ckpt) {
            const int kd = t;
            if (pfc_run_get_fields_f32(r, phi.data(), con.data()) != PFC_OK) return gpu_fail("checkpoint fields");
            if (misfit_phimax(r, o, phi, con, kd, scratch) != 0) return 2;
            if (!write_checkpoint_fields(o.outdir, kd, phi.data(), con.data(), L, M, N)) {
                cerr << "pfc-exp-cli: failed to write checkpoint files" << endl;
                return 2;
            }
            if (append_energy(r, o, kd) != 0) return 2;
            if (log.is_open()) {
                log << "step " << t << " timestamp_ms " << now_ms() << endl;
                log.flush();
            }
        }
    }
    return 0;
}

// ---------------------------------------------------------------------------
// CVD (CVD:111-203, 215-454)
// ---------------------------------------------------------------------------
void cvd_usage(const char *argv0) {
    cerr << "Usage: " << (argv0 ? argv0 : "pfc-exp-cli") << " --model cvd [options]\n"
         << "Options:\n"
         << "  --u0 <float>        Density/phi mean (default: 0.01)\n"
         << "  --con0 <float>      Concentration mean (default: 0.2)\n"
         << "  --sig <float>       Kernel decay sigma (default: 0.03)\n"
         << "  --dt <float>        Time step (default: 0.05)\n"
         << "  --dx <float>        Space step (default: 0.125)\n"
         << "  --steps <int>       Total iterations (default: 2000)\n"
         << "  --mod <int>         Output/analysis interval (default: 200)\n"
         << "  --seed <uint>       Random seed base (default: 20200604)\n"
         << "  --outdir <path>     Output directory (default: current dir)\n"
         << "  --grid <LxMxN>      Grid (default: 256x256x1)\n"
         << "  --precision <p>     mixed, fp32, fp64 or fp64-pure (default: mixed; fp64 on 3-D grids it does not take;\n"
         << "                      fp64 keeps the reference's own float roundings, so a run follows the reference's\n"
         << "                      trajectory, which FP32 storage leaves after ~100 steps at u0 0.01)\n"
         << "  --resume <kd>       Continue from checkpoint kd in --outdir\n"
         << "  -h, --help          Show this help\n";
}

// Lenient parser shared by CVD and Elastic (unknown options are skipped).
struct Lenient {
    int argc;
    char **argv;
    int i = 1;
};

int run_cvd_cli(int argc, char **argv) {
    SimOpts o;
    o.u0 = 0.01f;
    o.con0 = 0.2f;
    o.sig = 0.03f;
    o.dt = 0.05f;
    o.dx = 0.125f;
    o.axx = 0.0f;
    o.steps = 2000;
    o.mod = 200;
    o.seed = 20200604u;
    o.grainx = o.grainy = o.grainz = 1;
    for (int i = 1; i < argc; ++i) {
        if (!argv[i]) continue;
        if (strcmp(argv[i], "-h") == 0 || strcmp(argv[i], "--help") == 0) {
            cvd_usage(argv[0]);
            return 0;
        }
    }
    bool bad = false;
    for (int i = 1; i < argc && !bad; ++i) {
        const char *raw = argv[i];
        if (!raw) continue;
        std::string_view arg(raw);
        auto value = [&](const char *opt) -> const char * {
            if (arg == opt) {
                if (i + 1 >= argc) {
                    cerr << "Missing value after " << opt << "\n";
                    return nullptr;
                }
                return argv[++i];
            }
            return raw + strlen(opt) + 1;
        };
        auto is = [&](const char *opt) { return arg == opt || has_prefix(arg, std::string(opt) + "="); };
        if (is("--u0")) bad = !parse_float(value("--u0"), o.u0);
        else if (is("--con0")) bad = !parse_float(value("--con0"), o.con0);
        else if (is("--sig")) bad = !parse_float(value("--sig"), o.sig);
        else if (is("--dt")) bad = !parse_float(value("--dt"), o.dt);
        else if (is("--dx")) bad = !parse_float(value("--dx"), o.dx);
        else if (is("--steps")) bad = !parse_int(value("--steps"), o.steps);
        else if (is("--mod")) bad = !parse_int(value("--mod"), o.mod);
        else if (is("--seed")) bad = !parse_uint(value("--seed"), o.seed);
        else if (is("--grid")) bad = !parse_grid(value("--grid"), o.L, o.M, o.N);
        else if (is("--precision")) bad = !parse_precision(value("--precision"), o.precision);
        else if (is("--resume")) bad = !parse_int(value("--resume"), o.resume) || o.resume < 0;
        else if (is("--outdir")) {
            const char *v = value("--outdir");
            if (!v || *v == '\0') bad = true;
            else o.outdir = v;
        }
        // other options are skipped (CVD:192-193)
    }
    if (!bad && (o.steps <= 0 || o.dt <= 0.0f || o.dx <= 0.0f || o.mod <= 0)) {
        cerr << "Invalid parameter values\n";
        bad = true;
    }
    if (bad) {
        cvd_usage(argv[0]);
        return 2;
    }
    const int L = o.L, M = o.M, N = o.N;
    if (!setup_outdir(o.outdir)) return 2;
    cerr << "CVD Run config: "
         << "u0=" << o.u0 << " con0=" << o.con0 << " sig=" << o.sig << " dt=" << o.dt << " dx=" << o.dx
         << " steps=" << o.steps << " mod=" << o.mod << " seed=" << o.seed << " grid=(" << L << "," << M << "," << N
         << ")"
         << " outdir=" << (o.outdir.empty() ? "." : o.outdir) << endl;
    {
        std::ofstream c(opath(o.outdir, "run_config.txt"), std::ios::out | std::ios::trunc);
        if (c.is_open()) {
            c << "model cvd\n";
            c << "u0 " << o.u0 << "\n";
            c << "con0 " << o.con0 << "\n";
            c << "sig " << o.sig << "\n";
            c << "dt " << o.dt << "\n";
            c << "dx " << o.dx << "\n";
            c << "steps " << o.steps << "\n";
            c << "mod " << o.mod << "\n";
            c << "seed " << o.seed << "\n";
            c << "L " << L << "\n";
            c << "M " << M << "\n";
            c << "N " << N << "\n";
        }
    }
    std::ofstream log(opath(o.outdir, "checkpoint_timestamps.txt"),
                      std::ios::out | (o.resume >= 0 ? std::ios::app : std::ios::trunc));
    if (log.is_open() && o.resume < 0) log << "# Checkpoint timestamps - Step number and milliseconds since epoch" << endl;

    pfc_run_params p;
    pfc_default_params(PFC_MODEL_CVD, &p);
    p.L = L;
    p.M = M;
    p.N = N;
    p.u0 = o.u0;
    p.con0 = o.con0;
    p.sig = o.sig;
    p.dt = o.dt;
    p.dx = o.dx;
    p.seed = o.seed;
    p.precision = o.precision >= 0 ? o.precision : default_precision(p);
    RunGuard g;
    if (pfc_run_create(&p, &g.r) != PFC_OK) return gpu_fail("run setup");
    pfc_run *r = g.r;
    const long P = (long)L * M * N;
    std::vector<float> phi(P), con(P);
    DevScratch phi_dev, scratch;
    // CVD checkpoint kd holds the state after step kd + 1 (CVD:425)
    if (o.resume >= 0) {
        const int rc = resume_run(r, o, o.resume, o.resume + 1);
        if (rc != 0) return rc;
    }
    // ENERGYC2 runs every step (CVD:442): the steps up to the next checkpoint (or the
    // last step) run as one pfc_run_advance_energies call, whose per-step energies are
    // those of a step-by-step loop, read back with one synchronisation
    std::vector<double> es, ms;
    for (int t = o.resume >= 0 ? o.resume + 1 : 0; t < o.steps;) {
        const int next_kd = (t % o.mod) == 0 ? t : t + (o.mod - t % o.mod);
        const int last = std::min(std::min(next_kd, o.steps - 1), t + 1023);
        const int n = last - t + 1;
        es.resize(n);
        ms.resize(n);
        // a run whose fields went non-finite goes on, as the reference does (its files
        // then hold the NaN values)
        const int rc = pfc_run_advance_energies(r, n, es.data(), ms.data());
        if (rc != PFC_OK && rc != PFC_E_NONFINITE) return gpu_fail("time step");
        for (int i = t; i <= last; ++i) fprintf(stderr, "PFC_PROGRESS step=%d total=%d\n", i + 1, o.steps);
        fflush(stderr);
        for (int i = 0; i < n - 1; ++i) append_energy_line(o.outdir, t + i, es[i], ms[i]);
        t = last;
        if ((t % o.mod) == 0) {
            const int kd = t;
            if (pfc_run_get_fields_f32(r, phi.data(), con.data()) != PFC_OK) return gpu_fail("checkpoint fields");
            // atompositionCFGC2 + GR + Q6_GLO (CVD:427, 1067-1520) on the checkpoint's phi
            if (!phi_dev.ensure(P * sizeof(float)) ||
                cudaMemcpyAsync(phi_dev.p, phi.data(), P * sizeof(float), cudaMemcpyHostToDevice, r->stream) !=
                    cudaSuccess)
                return gpu_fail("CVD analysis upload");
            CvdAnalysis ca;
            if (cvd_analyze((const float *)phi_dev.p, L, M, N, o.dx, o.u0, kd, r->stream, scratch, ca) != PFC_OK)
                return gpu_fail("CVD analysis");
            write_cvd_files(o.outdir, L, M, N, o.dx, ca);
            if (!write_checkpoint_fields(o.outdir, kd, phi.data(), con.data(), L, M, N)) {
                cerr << "pfc-exp-cli: failed to write checkpoint files" << endl;
                return 2;
            }
            if (log.is_open()) {
                log << "step " << t << " timestamp_ms " << now_ms() << endl;
                log.flush();
            }
        }
        append_energy_line(o.outdir, t, es[n - 1], ms[n - 1]);
        ++t;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Elastic (ELA:30-74, 137-289, 304-521, 2802-3011)
// ---------------------------------------------------------------------------
void elastic_usage(const char *argv0) {
    cerr << "Usage: " << (argv0 ? argv0 : "pfc-exp-cli") << " --model elastic [options]\n"
         << "Options:\n"
         << "  --u0 <float>        Density/phi mean (default: 0.05)\n"
         << "  --con0 <float>      Concentration mean (default: 0.2)\n"
         << "  --sig <float>       Kernel decay sigma (default: 0.05)\n"
         << "  --dt <float>        Time step (default: 0.1)\n"
         << "  --dx <float>        Space step (default: 0.125)\n"
         << "  --steps <int>       Total iterations (default: 2002)\n"
         << "  --mod <int>         Output/analysis interval (default: 200)\n"
         << "  --seed <uint>       Random seed base (default: 20200604)\n"
         << "  --grainx <int>      Initial grains in x (default: 2)\n"
         << "  --grainy <int>      Initial grains in y (default: 2)\n"
         << "  --grainz <int>      Initial grains in z (default: 1)\n"
         << "  --benchel <float>   Neighbor cutoff for elastic analysis (default: 1.7)\n"
         << "  --input-dir <path>  Directory with pre-computed phi/con data\n"
         << "  --outdir <path>     Output directory (default: current dir)\n"
         << "  -h, --help          Show this help\n";
}

// One checkpoint of the Elastic analysis; returns the process exit code (0 = go on).
int elastic_checkpoint(int kd, const std::string &input_dir, const std::string &outdir, int gL, int gM, int gN, float dx,
                       float benchel, cudaStream_t st, DevScratch &scratch) {
    int L = gL, M = gM, N = gN;
    std::vector<float> phi, con;
    const std::string fphi = input_file(input_dir, "phi_", kd);
    if (!read_vti(fphi, L, M, N, phi)) {
        cerr << "can't open input file: " << fphi << endl;
        return 2;
    }
    int Lc = L, Mc = M, Nc = N;
    const std::string fcon = input_file(input_dir, "con_", kd);
    if (!read_vti(fcon, Lc, Mc, Nc, con)) {
        cerr << "can't open input file: " << fcon << endl;
        return 2;
    }
    ElasticResult res;
    if (elastic_analyze(phi.data(), L, M, N, dx, benchel, st, scratch, res) != PFC_OK) return gpu_fail("Elastic analysis");
    write_elastic_files(outdir, kd, res, cerr);
    return 0;
}

int run_elastic_cli(int argc, char **argv) {
    float u0 = 0.05f, con0 = 0.2f, sig = 0.05f, dt = 0.1f, dx = 0.125f, benchel = 1.7f;
    int steps = 2002, mod = 200, grainx = 2, grainy = 2, grainz = 1;
    unsigned int seed = 20200604u;
    int gL = 0, gM = 0, gN = 0;
    std::string outdir, input_dir;
    for (int i = 1; i < argc; ++i) {
        if (!argv[i]) continue;
        if (strcmp(argv[i], "-h") == 0 || strcmp(argv[i], "--help") == 0) {
            elastic_usage(argv[0]);
            return 0;
        }
    }
    bool bad = false;
    for (int i = 1; i < argc && !bad; ++i) {
        const char *raw = argv[i];
        if (!raw) continue;
        std::string_view arg(raw);
        auto value = [&](const char *opt) -> const char * {
            if (arg == opt) {
                if (i + 1 >= argc) {
                    cerr << "Missing value after " << opt << "\n";
                    return nullptr;
                }
                return argv[++i];
            }
            return raw + strlen(opt) + 1;
        };
        auto is = [&](const char *opt) { return arg == opt || has_prefix(arg, std::string(opt) + "="); };
        if (is("--u0")) bad = !parse_float(value("--u0"), u0);
        else if (is("--con0")) bad = !parse_float(value("--con0"), con0);
        else if (is("--sig")) bad = !parse_float(value("--sig"), sig);
        else if (is("--dt")) bad = !parse_float(value("--dt"), dt);
        else if (is("--dx")) bad = !parse_float(value("--dx"), dx);
        else if (is("--steps")) bad = !parse_int(value("--steps"), steps);
        else if (is("--mod")) bad = !parse_int(value("--mod"), mod);
        else if (is("--seed")) bad = !parse_uint(value("--seed"), seed);
        else if (is("--grainx")) bad = !parse_int(value("--grainx"), grainx);
        else if (is("--grainy")) bad = !parse_int(value("--grainy"), grainy);
        else if (is("--grainz")) bad = !parse_int(value("--grainz"), grainz);
        else if (is("--benchel")) bad = !parse_float(value("--benchel"), benchel);
        else if (is("--grid")) bad = !parse_grid(value("--grid"), gL, gM, gN);
        else if (is("--input-dir")) {
            const char *v = value("--input-dir");
            if (!v || *v == '\0') bad = true;
            else input_dir = v;
        } else if (is("--outdir")) {
            const char *v = value("--outdir");
            if (!v || *v == '\0') bad = true;
            else outdir = v;
        }
    }
    if (!bad && (steps <= 0 || dt <= 0.0f || dx <= 0.0f || mod <= 0)) {
        cerr << "Invalid parameter values\n";
        bad = true;
    }
    if (bad) {
        elastic_usage(argv[0]);
        return 2;
    }
    if (!input_dir.empty()) {
        std::error_code ec;
        const auto abs_input = std::filesystem::absolute(input_dir, ec);
        if (!ec) input_dir = abs_input.string();
    }
    if (!setup_outdir(outdir)) return 2;
    const int rL = gL > 0 ? gL : 256, rM = gM > 0 ? gM : 256, rN = gN > 0 ? gN : 1;
    cerr << "Elastic Run config: "
         << "u0=" << u0 << " con0=" << con0 << " sig=" << sig << " dt=" << dt << " dx=" << dx << " steps=" << steps
         << " mod=" << mod << " seed=" << seed << " grid=(" << rL << "," << rM << "," << rN << ")"
         << " grain=(" << grainx << "," << grainy << "," << grainz << ")"
         << " benchel=" << benchel << " input_dir=" << (input_dir.empty() ? "." : input_dir)
         << " outdir=" << (outdir.empty() ? "." : outdir) << endl;
    {
        std::ofstream c(opath(outdir, "run_config.txt"), std::ios::out | std::ios::trunc);
        if (c.is_open()) {
            c << "model elastic\n";
            c << "u0 " << u0 << "\n";
            c << "con0 " << con0 << "\n";
            c << "sig " << sig << "\n";
            c << "dt " << dt << "\n";
            c << "dx " << dx << "\n";
            c << "steps " << steps << "\n";
            c << "mod " << mod << "\n";
            c << "seed " << seed << "\n";
            c << "L " << rL << "\n";
            c << "M " << rM << "\n";
            c << "N " << rN << "\n";
            c << "grainx " << grainx << "\n";
            c << "grainy " << grainy << "\n";
            c << "grainz " << grainz << "\n";
            c << "benchel " << benchel << "\n";
            if (!input_dir.empty()) c << "input_dir " << input_dir << "\n";
        }
    }
    std::ofstream log(opath(outdir, "checkpoint_timestamps.txt"), std::ios::out | std::ios::trunc);
    if (log.is_open()) log << "# Checkpoint timestamps - Step number and milliseconds since epoch" << endl;
    int dev = 0;
    Context *ctx = nullptr;
    if (get_context(dev, &ctx) != PFC_OK) return gpu_fail("device setup");
    cudaSetDevice(dev);
    DevScratch scratch;
    const std::vector<int> ck = collect_steps(input_dir);
    if (!ck.empty()) {
        cerr << "Elastic detected " << ck.size() << " checkpoint step(s)";
        cerr << " [";
        const size_t shown = std::min<size_t>(ck.size(), 8);
        for (size_t i = 0; i < shown; ++i) {
            if (i) cerr << ", ";
            cerr << ck[i];
        }
        if (ck.size() > shown) cerr << ", ..., " << ck.back();
        cerr << "]";
        cerr << endl;
        for (size_t idx = 0; idx < ck.size(); ++idx) {
            fprintf(stderr, "PFC_PROGRESS step=%zu total=%zu\n", idx + 1, ck.size());
            fflush(stderr);
            const int rc = elastic_checkpoint(ck[idx], input_dir, outdir, gL, gM, gN, dx, benchel, ctx->stream, scratch);
            if (rc != 0) return rc;
        }
    } else {
        int total = 0;
        for (int t = 0; t < steps; t++)
            if (((t + 1) % mod) == 0 || t + 1 == steps) ++total;
        int done = 0;
        for (int t = 0; t < steps; t++) {
            const int s = t + 1;
            if ((s % mod) == 0 || s == steps) {
                ++done;
                fprintf(stderr, "PFC_PROGRESS step=%d total=%d\n", done, total);
                fflush(stderr);
                const int rc = elastic_checkpoint(s, input_dir, outdir, gL, gM, gN, dx, benchel, ctx->stream, scratch);
                if (rc != 0) return rc;
            }
        }
    }
    return 0;
}

void global_usage(const char *argv0) {
    cerr << "Usage: " << (argv0 ? argv0 : "pfc-exp-cli") << " [--model <name>] [model-options...]\n\n"
         << "Models:\n"
         << "  misfit    Phase-field crystal with misfit strain (default)\n"
         << "  cvd       Controlled vapor deposition / two-phase growth\n"
         << "  elastic   Post-processing: elastic strain & crystallographic order\n\n"
         << "Use --model <name> --help for model-specific options.\n"
         << "--batch <file.json> runs a whole parameter sweep (Fixed / Range / List per parameter)\n"
         << "on one GPU, each run in its own folder.\n";
}

}  // namespace

// main_cli.cpp:24-88
namespace {

// A value as the GUI hands it to pfc-exp-cli: QString::number(v, 'g', 10) on the
// command line (MainWindow.cpp:2402), read back with strtof.
float as_cli_float(double v) {
    char b[64];
    snprintf(b, sizeof(b), "%.10g", v);
    return strtof(b, nullptr);
}

// pfc-exp-cli --batch <file>: a whole GUI sweep (sweep.h) through the engine, each
// run writing into its own folder what pfc-exp-cli would write there.  Progress lines
// count finished runs.  Exit code 0 when every run finished, else 2.
int run_batch_cli(const std::string &path) {
    std::ifstream in(path);
    if (!in.is_open()) {
        cerr << "can't open batch file: " << path << endl;
        return 2;
    }
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    sweep::SweepSpec sp;
    std::string err;
    if (!sweep::parse_sweep(text, sp, err)) {
        cerr << "batch file " << path << ": " << err << endl;
        return 2;
    }
    pfc_engine_opts eo{};
    eo.hbm_budget_bytes = sp.budget_gb * 1e9;
    eo.max_active = sp.max_active;
    pfc_engine *eng = nullptr;
    if (pfc_engine_create(&eo, &eng) != PFC_OK) return gpu_fail("engine");
    const bool ela = sp.model == "elastic";
    const int model = sp.model == "cvd" ? PFC_MODEL_CVD : PFC_MODEL_MISFIT;
    int failed = 0, done = 0;
    const int total = (int)sp.runs.size();
    std::vector<uint64_t> ids;
    for (const auto &r : sp.runs) {
        std::string why;
        if (!make_dir(r.out_dir, &why)) {
            cerr << "Failed to create --outdir '" << r.out_dir << "': " << why << endl;
            ++failed;
            continue;
        }
        {
            std::ofstream pj(opath(r.out_dir, "params.json"), std::ios::out | std::ios::trunc);
            pj << sweep::params_json(sp, r);
        }
        pfc_job j{};
        pfc_default_params(model, &j.params);
        j.params.L = sp.L;
        j.params.M = sp.M;
        j.params.N = sp.N;
        j.params.u0 = as_cli_float(r.u0);
        j.params.con0 = as_cli_float(r.con0);
        j.params.sig = as_cli_float(r.sig);
        j.params.dt = as_cli_float(r.dt);
        j.params.dx = as_cli_float(r.dx);
        j.params.seed = r.seed;
        j.kind = ela ? PFC_JOB_ELASTIC : model;
        j.steps = r.steps;
        j.mod = r.mod;
        j.outdir = r.out_dir.c_str();
        j.input_dir = ela ? sp.input_dir.c_str() : nullptr;
        j.benchel = as_cli_float(r.benchel);
        uint64_t id = 0;
        if (pfc_submit(eng, &j, &id) != PFC_OK) {
            cerr << "run " << r.index << ": " << pfc_last_error() << endl;
            ++failed;
            continue;
        }
        ids.push_back(id);
    }
    std::vector<pfc_event> ev(64);
    size_t finished = 0;
    while (finished < ids.size()) {
        int n = 0;
        if (pfc_wait(eng, ev.data(), (int)ev.size(), &n, 1000) != PFC_OK) break;
        for (int i = 0; i < n; ++i) {
            const pfc_event &e = ev[i];
            if (e.type != PFC_EV_DONE && e.type != PFC_EV_FAILED && e.type != PFC_EV_CANCELLED) continue;
            ++finished;
            if (e.type == PFC_EV_DONE) ++done;
            else ++failed;
            cout << "PFC_PROGRESS step=" << done + failed << " total=" << total << endl;
        }
    }
    pfc_engine_destroy(eng);
    cerr << "batch: " << done << " of " << total << " runs finished" << (failed ? ", some failed" : "") << endl;
    return failed == 0 && done == total ? 0 : 2;
}

}  // namespace

extern "C" int pfc_run_cli(int argc, char **argv) {
    for (int i = 1; i + 1 < argc; ++i)
        if (argv[i] && std::string_view(argv[i]) == "--batch") return run_batch_cli(argv[i + 1]);
    for (int i = 1; i < argc; ++i)
        if (argv[i] && std::string_view(argv[i]).substr(0, 8) == "--batch=") return run_batch_cli(argv[i] + 8);
    std::string model = "misfit";
    std::vector<char *> nv;
    nv.push_back(argc > 0 ? argv[0] : (char *)"pfc-exp-cli");
    for (int i = 1; i < argc; ++i) {
        if (!argv[i]) continue;
        std::string_view arg(argv[i]);
        if (arg == "--model" || arg == "-m") {
            if (i + 1 < argc) {
                model = argv[++i];
            } else {
                cerr << "Missing value after --model\n";
                global_usage(argv[0]);
                return 2;
            }
            continue;
        }
        if (arg.substr(0, 8) == "--model=") {
            model = std::string(arg.substr(8));
            continue;
        }
        if (arg == "-h" || arg == "--help") {
            if (model == "misfit" && i == 1) {
                bool has_model = false;
                for (int j = i + 1; j < argc; ++j)
                    if (argv[j] &&
                        (std::string_view(argv[j]) == "--model" || std::string_view(argv[j]).substr(0, 8) == "--model=")) {
                        has_model = true;
                        break;
                    }
                if (!has_model) {
                    global_usage(argv[0]);
                    return 0;
                }
            }
        }
        nv.push_back(argv[i]);
    }
    const int nargc = (int)nv.size();
    nv.push_back(nullptr);
    if (model == "misfit") return run_misfit_cli(nargc, nv.data());
    if (model == "cvd") return run_cvd_cli(nargc, nv.data());
    if (model == "elastic") return run_elastic_cli(nargc, nv.data());
    cerr << "Unknown model: " << model << "\n";
    global_usage(argv[0]);
    return 2;
}

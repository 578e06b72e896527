// checkpoint.h -- checkpoint files and the Elastic analysis, shared by the
// pfc-exp-cli interface (cli.cpp) and the engine (serve.cpp), so that both write
// the same bytes.
//
// Formats restated from the reference (paths within zhiqing0205/PFC-Exp-GUI):
//   VTI / PVTI writers      src/experiment/misfit_uniform_time_seed_fftw_early.cpp:1588-1810
//   VTI reader              src/experiment/elastic.cpp:2562-2645
//   checkpoint discovery    src/experiment/elastic.cpp:37-74 (CollectAvailableCheckpointSteps)
//   Phimax_<kd>.txt         misfit_uniform_time_seed_fftw_early.cpp:3500-3556 (two lines per
//                           atom, z and z + 20), elastic.cpp:2990-3011 (one line per atom)
//   strain_<kd>.txt         elastic.cpp:3740-3776
//   q4q6_<kd>.txt           elastic.cpp:3330-3389
//   run_config.txt          misfit_uniform_time_seed_fftw_early.cpp:371-387, cvd.cpp:273-284
// Text values use std::fixed with precision(4), as the reference's streams do.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <ostream>
#include <set>
#include <string>
#include <vector>

#include "pfc_b200.h"

namespace pfc {
int phimax_misfit_dev(const float *d_phi, const float *d_con, int L, int M, float dx, float con0, double *d_out,
                      int cap, int *count, int *raw_count, cudaStream_t st);
int phimax_elastic_dev(const float *d_phi, int L, int M, int N, float dx, double *d_out, int cap, int *count,
                       cudaStream_t st);
int cvd_atoms_dev(const float *d_phi, int L, int M, int N, float dx, float u0, double *d_out, int cap, int *count,
                  float *stats_host, cudaStream_t st);
int cvd_gr_dev(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *hist,
               int maxbin, cudaStream_t st);
int cvd_q6_dev(const float *x, const float *y, const float *z, int n, int L, int M, int N, float dx, unsigned *nb,
               float *ql, float *ql_global_host, cudaStream_t st);

namespace ckpt {

inline std::string opath(const std::string &dir, const std::string &name) {
    return dir.empty() ? name : (std::filesystem::path(dir) / name).string();
}

inline long long now_ms() {
    return std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::system_clock::now().time_since_epoch())
        .count();
}

// Create an output directory (and its parents); false if it cannot be a directory.
inline bool make_dir(const std::string &dir, std::string *why = nullptr) {
    if (dir.empty()) return true;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) {
        if (why) *why = ec.message();
        return false;
    }
    if (!std::filesystem::is_directory(dir, ec)) {
        if (why) *why = "Not a directory";
        return false;
    }
    return true;
}

// Device scratch that grows on demand.
struct DevScratch {
    void *p = nullptr;
    size_t bytes = 0;
    DevScratch() = default;
    DevScratch(const DevScratch &) = delete;
    DevScratch &operator=(const DevScratch &) = delete;
    ~DevScratch() {
        if (p) cudaFree(p);
    }
    bool ensure(size_t b) {
        if (b <= bytes) return true;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, b) != cudaSuccess) return false;
        bytes = b;
        return true;
    }
};

// ---------------------------------------------------------------------------
// VTI / PVTI.  data: field in layout n + N*(m + M*l); written as Float32 with l fastest.
// ---------------------------------------------------------------------------
inline bool write_vti(const std::string &path, const char *name, const float *data, int L, int M, int N) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return false;
    const int startn = 0, endn = L - 1;
    const int bytes = (int)((long)N * M * L * (long)sizeof(float) + (long)sizeof(int));
    fprintf(f, "<?xml version=\"1.0\"?>\n");
    fprintf(f, "<VTKFile type=\"ImageData\" version=\"0.1\"  byte_order=\"LittleEndian\">\n");
    fprintf(f, "<ImageData WholeExtent=\"%d %d %d %d %d %d\"   Origin=\"%d %d %d\" Spacing=\"%d %d %d\">\n", startn, endn,
            0, M - 1, 0, N - 1, 0, 0, 0, 1, 1, 1);
    fprintf(f, "<Piece Extent=\"%d %d %d %d %d %d\">\n", startn, endn, 0, M - 1, 0, N - 1);
    fprintf(f, "<PointData Scalars=\"%s\">\n", name);
    fprintf(f, "<DataArray type=\"Float32\" Name=\"%s\"   format=\"appended\" offset=\"%d\" />\n", name, 0);
    fprintf(f, "</PointData>\n");
    fprintf(f, "<CellData>\n");
    fprintf(f, "</CellData>\n");
    fprintf(f, "</Piece>\n");
    fprintf(f, "</ImageData>\n");
    fprintf(f, "<AppendedData encoding=\"raw\">\n");
    fprintf(f, "_");
    fwrite(&bytes, sizeof(int), 1, f);
    std::vector<float> out((size_t)L * M * N);
    size_t o = 0;
    for (int n = 0; n < N; n++)
        for (int m = 0; m < M; m++)
            for (int l = 0; l < L; l++) out[o++] = data[n + (long)N * (m + (long)M * l)];
    fwrite(out.data(), sizeof(float), out.size(), f);
    fprintf(f, "\n");
    fprintf(f, "</AppendedData>\n");
    fprintf(f, "</VTKFile>\n");
    return fclose(f) == 0;
}

inline void write_pvti(const std::string &path, const char *name, const std::string &prefix, int kd, int L, int M,
                       int N) {
    std::ofstream o(path, std::ios_base::out);
    o.setf(std::ios_base::fixed, std::ios_base::floatfield);
    o.precision(4);
    o << "<?xml version=\"1.0\"?>" << std::endl;
    o << "<VTKFile type=\"PImageData\" version=\"0.1\" byte_order=\"LittleEndian\">" << std::endl;
    o << "  <PImageData WholeExtent=\"0 " << L - 1 << " 0 " << M - 1 << " " << 0 << " " << N - 1
      << "\" GhostLevel=\"#\" Origin=\"0  0  0\"  Spacing=\"1  1  1\">" << std::endl;
    o << "    <PPointData>" << std::endl;
    o << "      <PDataArray type=\"Float32\" Name=\"" << name << "\"/>" << std::endl;
    o << "    </PPointData>" << std::endl;
    o << "    <Piece Extent=\"0 " << L - 1 << " 0 " << M - 1 << " " << 0 << " " << N - 1 << "\" Source=\"" << prefix
      << kd << "_0.vti\"/>" << std::endl;
    o << "  </PImageData>" << std::endl;
    o << "</VTKFile>" << std::endl;
}

inline bool write_checkpoint_fields(const std::string &outdir, int kd, const float *phi, const float *con, int L, int M,
                                    int N) {
    char fn[64];
    snprintf(fn, sizeof(fn), "phi_%d_%d.vti", kd, 0);
    if (!write_vti(opath(outdir, fn), "phi", phi, L, M, N)) return false;
    snprintf(fn, sizeof(fn), "phi_%d.pvti", kd);
    write_pvti(opath(outdir, fn), "phi", "phi_", kd, L, M, N);
    snprintf(fn, sizeof(fn), "con_%d_%d.vti", kd, 0);
    if (!write_vti(opath(outdir, fn), "con", con, L, M, N)) return false;
    snprintf(fn, sizeof(fn), "con_%d.pvti", kd);
    write_pvti(opath(outdir, fn), "con", "con_", kd, L, M, N);
    return true;
}

// VTI reader: 12 header lines, '_', int32 byte count, then Float32 values with l
// fastest.  The grid comes from WholeExtent unless L > 0 is given.
inline bool read_vti(const std::string &path, int &L, int &M, int &N, std::vector<float> &field) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    char buf[100];
    int gl = -1, gm = -1, gn = -1;
    for (int i = 1; i < 13; ++i) {
        if (!fgets(buf, sizeof(buf), f)) break;
        int a, b, c, d, e, g;
        const char *w = strstr(buf, "WholeExtent=\"");
        if (w && sscanf(w + 13, "%d %d %d %d %d %d", &a, &b, &c, &d, &e, &g) == 6 && gl < 0) {
            gl = b - a + 1;
            gm = d - c + 1;
            gn = g - e + 1;
        }
    }
    (void)fgetc(f);
    int bytes = 0;
    if (fread(&bytes, sizeof(int), 1, f) != 1) {
        fclose(f);
        return false;
    }
    if (L <= 0) {
        L = gl;
        M = gm;
        N = gn;
    }
    if (L <= 0 || M <= 0 || N <= 0) {
        fclose(f);
        return false;
    }
    const long P = (long)L * M * N;
    std::vector<float> raw(P, 0.0f);
    const size_t got = fread(raw.data(), sizeof(float), P, f);
    fclose(f);
    (void)got;  // a short file leaves the remaining values 0, as the reference's unchecked reads do
    field.assign(P, 0.0f);
    long o = 0;
    for (int n = 0; n < N; n++)
        for (int m = 0; m < M; m++)
            for (int l = 0; l < L; l++) field[n + (long)N * (m + (long)M * l)] = raw[o++];
    return true;
}

inline std::string input_file(const std::string &input_dir, const char *prefix, int step) {
    char fn[64];
    snprintf(fn, sizeof(fn), "%s%d%s%d%s", prefix, step, "_", 0, ".vti");
    if (input_dir.empty()) return std::string(fn);
    return (std::filesystem::path(input_dir) / fn).string();
}

// Steps with both phi_<s>_<r>.vti and con_<s>_<r>.vti, ascending; step 0 is dropped
// when a later step exists.
inline std::vector<int> collect_steps(const std::string &input_dir) {
    std::vector<int> out;
    const std::filesystem::path dir = input_dir.empty() ? std::filesystem::current_path() : std::filesystem::path(input_dir);
    std::error_code ec;
    if (!std::filesystem::exists(dir, ec) || ec) return out;
    std::set<int> ps, cs;
    for (const auto &e : std::filesystem::directory_iterator(dir, ec)) {
        if (ec) break;
        if (!e.is_regular_file()) continue;
        const std::string name = e.path().filename().string();
        int step = 0, rank = 0;
        if (sscanf(name.c_str(), "phi_%d_%d.vti", &step, &rank) == 2) {
            ps.insert(step);
            continue;
        }
        if (sscanf(name.c_str(), "con_%d_%d.vti", &step, &rank) == 2) cs.insert(step);
    }
    bool has_positive = false;
    for (int s : ps) {
        if (!cs.count(s)) continue;
        if (s > 0) has_positive = true;
        out.push_back(s);
    }
    std::sort(out.begin(), out.end());
    if (has_positive) out.erase(std::remove(out.begin(), out.end(), 0), out.end());
    return out;
}

// ---------------------------------------------------------------------------
// Misfit Phimax_<kd>.txt from the peak finder's records (x, y, z, phimax, con);
// records with a non-finite value or x < 0 are skipped.  Returns the atoms written.
// ---------------------------------------------------------------------------
inline bool misfit_atom_ok(const double *a) {
    return std::isfinite(a[0]) && std::isfinite(a[1]) && std::isfinite(a[2]) && std::isfinite(a[3]) &&
           std::isfinite(a[4]) && a[0] >= 0;
}
inline int count_misfit_atoms(const std::vector<double> &atoms, int count) {
    int total = 0;
    for (int i = 0; i < count; ++i) total += misfit_atom_ok(&atoms[(size_t)i * 5]) ? 1 : 0;
    return total;
}
inline int write_phimax_misfit(const std::string &outdir, int kd, const std::vector<double> &atoms, int count) {
    const int total = count_misfit_atoms(atoms, count);
    char fn[64];
    snprintf(fn, sizeof(fn), "Phimax_%d.txt", kd);
    std::ofstream f(opath(outdir, fn), std::ios_base::out);
    f.setf(std::ios_base::fixed, std::ios_base::floatfield);
    f.precision(4);
    f << 2 * total << std::endl;
    f << "Kommentar" << std::endl;
    for (int i = 0; i < count; ++i) {
        const double *a = &atoms[(size_t)i * 5];
        if (!misfit_atom_ok(a)) continue;
        f << a[0] << " " << a[1] << " " << a[2] << " " << a[3] << " " << a[4] << std::endl;
        f << a[0] << " " << a[1] << " " << a[2] + 20 << " " << a[3] << " " << a[4] << std::endl;
    }
    return total;
}

inline void append_energy_line(const std::string &outdir, int kd, double e, double d) {
    std::ofstream f(opath(outdir, "energy.txt"), std::ios_base::out | std::ios_base::app);
    f << kd << " " << e << " " << d << std::endl;
}

// run_config.txt of a Misfit or CVD run (the CVD file has no grain/noise lines).
inline void write_run_config(const std::string &outdir, const pfc_run_params &p, int steps, int mod) {
    std::ofstream c(opath(outdir, "run_config.txt"), std::ios::out | std::ios::trunc);
    if (!c.is_open()) return;
    c << (p.model == PFC_MODEL_CVD ? "model cvd\n" : "model misfit\n");
    c << "u0 " << p.u0 << "\n";
    c << "con0 " << p.con0 << "\n";
    c << "sig " << p.sig << "\n";
    c << "dt " << p.dt << "\n";
    c << "dx " << p.dx << "\n";
    c << "steps " << steps << "\n";
    c << "mod " << mod << "\n";
    c << "seed " << p.seed << "\n";
    c << "L " << p.L << "\n";
    c << "M " << p.M << "\n";
    c << "N " << p.N << "\n";
    if (p.model == PFC_MODEL_CVD) return;
    const float b0 = (p.dx > 0.0f && p.dt > 0.0f && p.axx >= 0.0f)
                         ? (float)std::sqrt(p.axx / p.dx / p.dx / p.dx / p.dt)
                         : 0.0f;
    c << "grainx " << p.grainx << "\n";
    c << "grainy " << p.grainy << "\n";
    c << "grainz " << p.grainz << "\n";
    c << "axx " << p.axx << "\n";
    c << "b0 " << b0 << "\n";
}

// ---------------------------------------------------------------------------
// Elastic analysis of one field (ELA:2802-3011, 3586-3776, 3013-3389): Phimax atoms,
// strain and neighbour counts, q4 / q6.
// ---------------------------------------------------------------------------
struct ElasticResult {
    int n = 0;                          // atoms found (records, including skipped ones)
    std::vector<double> atoms;          // 4 per atom: x, y, z, phimax
    std::vector<double> x, y, z, strain, q4, q6;
    std::vector<uint32_t> nb;
};

// Returns PFC_OK or a PFC_E_* code (pfc_last_error describes it).
inline int elastic_analyze(const float *phi, int L, int M, int N, float dx, float benchel, cudaStream_t st,
                           DevScratch &scratch, ElasticResult &r) {
    const long P = (long)L * M * N;
    const long cap = P + 1;
    if (!scratch.ensure(P * sizeof(float) + 256 + cap * 4 * sizeof(double))) return PFC_E_NOMEM;
    float *dphi = (float *)scratch.p;
    double *datoms = (double *)((char *)scratch.p + ((P * sizeof(float) + 255) / 256) * 256);
    if (cudaMemcpyAsync(dphi, phi, P * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess) return PFC_E_CUDA;
    int n = 0;
    int rc = phimax_elastic_dev(dphi, L, M, N, dx, datoms, (int)cap, &n, st);
    if (rc != PFC_OK) return rc;
    r.n = n;
    r.atoms.assign((size_t)n * 4, 0.0);
    if (n > 0 && cudaMemcpyAsync(r.atoms.data(), datoms, r.atoms.size() * sizeof(double), cudaMemcpyDeviceToHost, st) !=
                     cudaSuccess)
        return PFC_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PFC_E_CUDA;
    r.x.resize(n);
    r.y.resize(n);
    r.z.resize(n);
    for (int i = 0; i < n; ++i) {
        r.x[i] = r.atoms[4 * i];
        r.y[i] = r.atoms[4 * i + 1];
        r.z[i] = r.atoms[4 * i + 2];
    }
    r.strain.assign(n, 0.0);
    r.q4.assign(n, 0.0);
    r.q6.assign(n, 0.0);
    r.nb.assign(n, 0u);
    if (n > 0) {
        rc = pfc_elastic3d(r.x.data(), r.y.data(), r.z.data(), n, L, M, N, dx, benchel, r.strain.data(), r.nb.data());
        if (rc != PFC_OK) return rc;
        rc = pfc_cryst_order(r.x.data(), r.y.data(), r.z.data(), n, L, M, N, dx, r.q4.data(), r.q6.data());
        if (rc != PFC_OK) return rc;
    }
    return PFC_OK;
}

// Phimax_<kd>.txt, strain_<kd>.txt and q4q6_<kd>.txt of one Elastic checkpoint; the
// reference's q4q6 diagnostic line goes to diag.  Returns the atoms written.
inline int write_elastic_files(const std::string &outdir, int kd, const ElasticResult &r, std::ostream &diag) {
    const int n = r.n;
    char fn[64];
    {
        snprintf(fn, sizeof(fn), "Phimax_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        f << n << std::endl;
        f << "Kommentar" << std::endl;
        for (int i = 0; i < n; ++i)
            if (r.x[i] >= 0) f << r.x[i] << " " << r.y[i] << " " << r.z[i] << " " << r.atoms[4 * i + 3] << std::endl;
    }
    {
        snprintf(fn, sizeof(fn), "strain_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        f << n << std::endl;
        f << "Kommentar" << std::endl;
        for (int i = 0; i < n; ++i)
            if (r.x[i] >= 0)
                f << "st" << " " << r.x[i] << " " << r.y[i] << " " << r.z[i] << " " << r.strain[i] << " " << r.nb[i]
                  << std::endl;
    }
    int total = 0;
    for (int i = 0; i < n; ++i)
        if (r.x[i] >= 0) total++;
    snprintf(fn, sizeof(fn), "q4q6_%d.txt", kd);
    std::ofstream f(opath(outdir, fn), std::ios_base::out);
    f.setf(std::ios_base::fixed, std::ios_base::floatfield);
    f.precision(4);
    f << total << std::endl;
    f << "Kommentar" << std::endl;
    double qMinX = 1e30, qMaxX = -1e30, qMinY = 1e30, qMaxY = -1e30;
    for (int i = 0; i < n; ++i) {
        if (r.x[i] >= 0) {
            f << "qc" << " " << r.x[i] << " " << r.y[i] << " " << r.z[i] << " " << r.q4[i] << " " << r.q6[i]
              << std::endl;
            if (r.x[i] < qMinX) qMinX = r.x[i];
            if (r.x[i] > qMaxX) qMaxX = r.x[i];
            if (r.y[i] < qMinY) qMinY = r.y[i];
            if (r.y[i] > qMaxY) qMaxY = r.y[i];
        }
    }
    diag << "q4q6_" << kd << ".txt: atoms=" << total << " x=[" << qMinX << "," << qMaxX << "] y=[" << qMinY << ","
         << qMaxY << "]" << std::endl;
    return total;
}

// ---------------------------------------------------------------------------
// CVD checkpoint analysis (CVD:1067-1520): atompositionCFGC2's peak finder, GR, and
// Q6_GLO at checkpoints with kd % 20 == 0.  The pair work runs on the GPU; the files
// are formatted here with the reference's float arithmetic.
// ---------------------------------------------------------------------------
struct CvdAnalysis {
    int kd = 0;
    float phic = 0.f, phimax = 0.f;
    int count = 0;             // records, including a (-1, -1, -1) "no atoms" record
    std::vector<float> rec;    // 4 per record: pc_x, pc_y, pc_z, pc_phi
    std::vector<unsigned> hist;
    bool q6 = false;
    std::vector<unsigned> nb;
    std::vector<float> ql;
    float ql_global = 0.f;
};

inline float cvd_delr() { return (float)(1.0f / 25.); }
inline int cvd_maxbin(int L, float dx) { return (int)(((float)L * dx) / cvd_delr()); }

// d_phi: device float field (layout n + N*(m + M*l)).
inline int cvd_analyze(const float *d_phi, int L, int M, int N, float dx, float u0, int kd, cudaStream_t st,
                       DevScratch &scratch, CvdAnalysis &r) {
    const long P = (long)L * M * N;
    const long cap = P + 1;
    const int maxbin = cvd_maxbin(L, dx);
    const size_t rec_bytes = ((size_t)cap * 4 * sizeof(double) + 255) / 256 * 256;
    const size_t xyz_bytes = ((size_t)3 * cap * sizeof(float) + 255) / 256 * 256;
    const size_t hist_bytes = ((size_t)(maxbin > 0 ? maxbin : 1) * sizeof(unsigned) + 255) / 256 * 256;
    const size_t q_bytes = (size_t)cap * (sizeof(unsigned) + sizeof(float)) + 256;
    if (!scratch.ensure(rec_bytes + xyz_bytes + hist_bytes + q_bytes)) return PFC_E_NOMEM;
    char *base = (char *)scratch.p;
    double *d_rec = (double *)base;
    float *d_xyz = (float *)(base + rec_bytes);
    unsigned *d_hist = (unsigned *)(base + rec_bytes + xyz_bytes);
    unsigned *d_nb = (unsigned *)(base + rec_bytes + xyz_bytes + hist_bytes);
    float *d_ql = (float *)(d_nb + cap);
    r.kd = kd;
    float stats[2];
    int found = 0;
    int rc = cvd_atoms_dev(d_phi, L, M, N, dx, u0, d_rec, (int)cap, &found, stats, st);
    if (rc != PFC_OK) return rc;
    r.phic = stats[0];
    r.phimax = stats[1];
    std::vector<double> rec((size_t)found * 4);
    if (found > 0 &&
        cudaMemcpyAsync(rec.data(), d_rec, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return PFC_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return PFC_E_CUDA;
    r.count = found > 0 ? found : 1;
    r.rec.assign((size_t)r.count * 4, 0.f);
    for (size_t i = 0; i < rec.size(); ++i) r.rec[i] = (float)rec[i];
    if (found == 0) r.rec[0] = r.rec[1] = r.rec[2] = -1.0f;  // CVD:1169
    const int n = r.count;
    std::vector<float> xyz((size_t)3 * n);
    for (int i = 0; i < n; ++i) {
        xyz[i] = r.rec[4 * i];
        xyz[n + i] = r.rec[4 * i + 1];
        xyz[2 * n + i] = r.rec[4 * i + 2];
    }
    if (cudaMemcpyAsync(d_xyz, xyz.data(), xyz.size() * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return PFC_E_CUDA;
    rc = cvd_gr_dev(d_xyz, d_xyz + n, d_xyz + 2 * n, n, L, M, N, dx, d_hist, maxbin, st);
    if (rc != PFC_OK) return rc;
    r.hist.assign(maxbin > 0 ? maxbin : 0, 0u);
    if (maxbin > 0 &&
        cudaMemcpyAsync(r.hist.data(), d_hist, maxbin * sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return PFC_E_CUDA;
    r.q6 = kd >= 0 && kd % 20 == 0;  // CVD:1254
    if (r.q6) {
        rc = cvd_q6_dev(d_xyz, d_xyz + n, d_xyz + 2 * n, n, L, M, N, dx, d_nb, d_ql, &r.ql_global, st);
        if (rc != PFC_OK) return rc;
        r.nb.assign(n, 0u);
        r.ql.assign(n, 0.f);
        if (cudaMemcpyAsync(r.nb.data(), d_nb, n * sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaMemcpyAsync(r.ql.data(), d_ql, n * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return PFC_E_CUDA;
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return PFC_E_CUDA;
    return PFC_OK;
}

// phimax.txt (appended), phiball_<kd>.cfg, Phimax_<kd>.txt, hist_<kd>.txt, Grq6_<kd>.txt
// and, with Q6, Ql_<kd>.txt and HistQ_<kd>.txt, as rank 0 of the reference writes them.
inline void write_cvd_files(const std::string &outdir, int L, int M, int N, float dx, const CvdAnalysis &r) {
    const int kd = r.kd;
    const float frame_x = (float)L * dx, frame_y = (float)M * dx, frame_z = (float)N * dx;
    {
        std::ofstream o(opath(outdir, "phimax.txt"), std::ios_base::out | std::ios_base::app);
        o << kd << " , " << r.phic << " , " << r.phimax << " , " << 0 << std::endl;
        o << "phimax is done" << " " << "myid=" << 0 << std::endl;
        o << " buf is done " << std::endl;
        o << " pc_xyz is initializing " << std::endl;
        o << " pc_xyz is done " << std::endl;
        o << " pc_xyz has been gathered " << std::endl;
    }
    const int n = r.count;
    int total = 0;
    for (int i = 0; i < n; ++i) total += r.rec[4 * i] >= 0 ? 1 : 0;
    char fn[64];
    {
        snprintf(fn, sizeof(fn), "phiball_%d.cfg", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        const float ai = 10.0f;
        f << "Number of particles = " << total << std::endl;
        f << "A = " << ai << " Angstrom (basic length-scale)" << std::endl;
        f << "H0(1,1) = " << frame_y << " A " << std::endl;
        f << "H0(1,2) = " << 0 << " A " << std::endl;
        f << "H0(1,3) = " << 0 << " A " << std::endl;
        f << "H0(2,1) = " << 0 << " A " << std::endl;
        f << "H0(2,2) = " << frame_z << " A " << std::endl;
        f << "H0(2,3) = " << 0 << " A " << std::endl;
        f << "H0(3,1) = " << 0 << " A " << std::endl;
        f << "H0(3,2) = " << 0 << " A " << std::endl;
        f << "H0(3,3) = " << frame_x << " A " << std::endl;
        f << ".NO_VELOCITY." << std::endl;
        f << "entry_count = 3" << std::endl;
        f << "63.546" << std::endl;
        f << "Cu" << std::endl;
        for (int i = 0; i < n; ++i)
            if (r.rec[4 * i] >= 0) f << r.rec[4 * i] << " " << r.rec[4 * i + 1] << " " << r.rec[4 * i + 2] << std::endl;
    }
    {
        snprintf(fn, sizeof(fn), "Phimax_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        f << total << std::endl;
        f << "Kommentar" << std::endl;
        for (int i = 0; i < n; ++i)
            if (r.rec[4 * i] >= 0)
                f << r.rec[4 * i + 2] * frame_x << " " << r.rec[4 * i] * frame_y << " " << r.rec[4 * i + 1] * frame_z
                  << " " << r.rec[4 * i + 3] << std::endl;
    }
    const int maxbin = (int)r.hist.size();
    {
        snprintf(fn, sizeof(fn), "hist_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        for (int ii = 0; ii < maxbin; ii++) f << ii << " " << r.hist[ii] << " " << maxbin << std::endl;
    }
    {
        const float delr = cvd_delr();
        const float rho = float(total) / float((float)(L * M * N) * dx * dx * dx);
        const float preco = (float)(4. * 3.1415926 * rho / 3.);
        snprintf(fn, sizeof(fn), "Grq6_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(4);
        for (int jj = 0; jj < maxbin; jj++) {
            const float rlower = float(jj) * delr;
            const float rupper = rlower + delr;
            const float nideal = preco * (rupper * rupper * rupper - rlower * rlower * rlower);
            const float gr = float(r.hist[jj]) / float(1) / float(total) / nideal;
            f << jj * delr << " " << gr << " " << r.hist[jj] << " " << nideal << std::endl;
        }
    }
    if (!r.q6) return;
    const float delq = 0.05f;
    unsigned histq[30] = {0};
    {
        snprintf(fn, sizeof(fn), "Ql_%d.txt", kd);
        std::ofstream f(opath(outdir, fn), std::ios_base::out);
        f.setf(std::ios_base::fixed, std::ios_base::floatfield);
        f.precision(6);
        for (int i = 0; i < n; i++) {
            f << i << " " << r.nb[i] << " " << r.ql[i] << " " << r.ql_global << std::endl;
            const unsigned bin = (unsigned)(int)(r.ql[i] / delq);
            if (bin < 30) histq[bin] = histq[bin] + 1;
        }
    }
    snprintf(fn, sizeof(fn), "HistQ_%d.txt", kd);
    std::ofstream f(opath(outdir, fn), std::ios_base::out);
    f.setf(std::ios_base::fixed, std::ios_base::floatfield);
    f.precision(4);
    for (int i = 0; i < 30; i++) f << (i + 1) * delq << " " << histq[i] << std::endl;
}

}  // namespace ckpt
}  // namespace pfc

// sweep.h -- the GUI's parameter sweeps as a batch file for pfc-exp-cli --batch.
//
// The GUI expands a sweep (each parameter Fixed, Range or List) into one run per
// combination and starts pfc-exp-cli once per run (src/gui/MainWindow.cpp:2632-2797:
// buildExperimentJobs; 2473-2560: makeDoubleRange / makeIntRange / list parsing;
// 2430-2471: params.json).  The batch file states the same sweep:
//
//   { "model": "misfit" | "cvd" | "elastic",
//     "out_dir": "<experiment root>",            // runs go to run_0001 ... (or the root, one run)
//     "grid": [L, M, N],                         // optional, default [256, 256, 1]
//     "params": { "u0": 0.05,                    // Fixed
//                 "con0": {"range": [0.1, 0.4, 0.1]},   // Range: start, end, step
//                 "seed": {"list": [1, 2, 3]} },        // List
//     "input_dir": "...", "benchel": 1.7,        // Elastic
//     "hbm_budget_gb": 150, "max_active": 0 }    // engine admission (optional)
//
// Parameters are expanded in the GUI's order (u0, con0, sig, dt, dx, steps, mod, seed,
// benchel), the last one changing fastest.  Each run folder gets the GUI's params.json.
#pragma once

#include <charconv>
#include <cmath>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace pfc {
namespace sweep {

// ---------------------------------------------------------------------------
// Minimal JSON reader (objects, arrays, numbers, strings, true / false / null).
// ---------------------------------------------------------------------------
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    bool integral = false;  // the number was written without fraction or exponent
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;
    const Json *get(const std::string &k) const {
        for (const auto &kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

class Parser {
  public:
    explicit Parser(const std::string &s) : s_(s) {}
    bool parse(Json &out, std::string &err) {
        if (!value(out, err)) return false;
        ws();
        if (i_ != s_.size()) return fail(err, "trailing characters");
        return true;
    }

  private:
    const std::string &s_;
    size_t i_ = 0;
    bool fail(std::string &err, const char *what) {
        err = std::string(what) + " at offset " + std::to_string(i_);
        return false;
    }
    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }
    bool lit(const char *w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(i_, n, w) != 0) return false;
        i_ += n;
        return true;
    }
    bool string(std::string &out, std::string &err) {
        if (s_[i_] != '"') return fail(err, "expected string");
        ++i_;
        out.clear();
        while (i_ < s_.size() && s_[i_] != '"') {
            char c = s_[i_++];
            if (c == '\\') {
                if (i_ >= s_.size()) return fail(err, "bad escape");
                char e = s_[i_++];
                switch (e) {
                    case 'n': c = '\n'; break;
                    case 't': c = '\t'; break;
                    case 'r': c = '\r'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'u': return fail(err, "\\u escapes are not supported");
                    default: c = e;
                }
            }
            out.push_back(c);
        }
        if (i_ >= s_.size()) return fail(err, "unterminated string");
        ++i_;
        return true;
    }
    bool value(Json &v, std::string &err) {
        ws();
        if (i_ >= s_.size()) return fail(err, "unexpected end");
        const char c = s_[i_];
        if (c == '{') {
            v.kind = Json::Object;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == '}') {
                ++i_;
                return true;
            }
            for (;;) {
                ws();
                std::string k;
                if (i_ >= s_.size() || !string(k, err)) return i_ >= s_.size() ? fail(err, "unexpected end") : false;
                ws();
                if (i_ >= s_.size() || s_[i_] != ':') return fail(err, "expected ':'");
                ++i_;
                Json x;
                if (!value(x, err)) return false;
                v.obj.emplace_back(k, std::move(x));
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == '}') {
                    ++i_;
                    return true;
                }
                return fail(err, "expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Array;
            ++i_;
            ws();
            if (i_ < s_.size() && s_[i_] == ']') {
                ++i_;
                return true;
            }
            for (;;) {
                Json x;
                if (!value(x, err)) return false;
                v.arr.push_back(std::move(x));
                ws();
                if (i_ < s_.size() && s_[i_] == ',') {
                    ++i_;
                    continue;
                }
                if (i_ < s_.size() && s_[i_] == ']') {
                    ++i_;
                    return true;
                }
                return fail(err, "expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            return string(v.str, err);
        }
        if (lit("true")) {
            v.kind = Json::Bool;
            v.b = true;
            return true;
        }
        if (lit("false")) {
            v.kind = Json::Bool;
            return true;
        }
        if (lit("null")) return true;
        const size_t start = i_;
        if (i_ < s_.size() && (s_[i_] == '-' || s_[i_] == '+')) ++i_;
        bool frac = false;
        while (i_ < s_.size() && (isdigit((unsigned char)s_[i_]) || s_[i_] == '.' || s_[i_] == 'e' || s_[i_] == 'E' ||
                                  ((s_[i_] == '-' || s_[i_] == '+') && (s_[i_ - 1] == 'e' || s_[i_ - 1] == 'E')))) {
            if (s_[i_] == '.' || s_[i_] == 'e' || s_[i_] == 'E') frac = true;
            ++i_;
        }
        if (i_ == start) return fail(err, "unexpected character");
        const std::string t = s_.substr(start, i_ - start);
        char *end = nullptr;
        v.num = strtod(t.c_str(), &end);
        if (!end || *end != '\0') return fail(err, "bad number");
        v.kind = Json::Number;
        v.integral = !frac;
        return true;
    }
};

// ---------------------------------------------------------------------------
// Sweep expansion
// ---------------------------------------------------------------------------
struct RunSpec {
    double u0, con0, sig, dt, dx, benchel;
    int steps, mod;
    unsigned seed;
    int index = 1, total = 1;
    std::string out_dir;
};

struct SweepSpec {
    std::string model = "misfit";
    std::string out_dir, input_dir;
    int L = 256, M = 256, N = 1;
    double budget_gb = 0.0;
    int max_active = 0;
    std::vector<RunSpec> runs;
};

// Values of one parameter: a number (Fixed), {"range": [start, end, step]} or
// {"list": [...]}, with the GUI's range rules (MainWindow.cpp:2473-2510).
inline bool param_values(const Json &v, bool is_int, std::vector<double> &out, std::string &err) {
    out.clear();
    if (v.kind == Json::Number) {
        out.push_back(v.num);
        return true;
    }
    if (v.kind != Json::Object) {
        err = "expected a number, {\"range\": [...]} or {\"list\": [...]}";
        return false;
    }
    if (const Json *r = v.get("range")) {
        if (r->kind != Json::Array || r->arr.size() != 3) {
            err = "range needs [start, end, step]";
            return false;
        }
        const double a = r->arr[0].num, b = r->arr[1].num, st = r->arr[2].num;
        if (!(st > 0)) {
            err = "Step must be > 0.";
            return false;
        }
        if (b < a) {
            err = "End must be >= start.";
            return false;
        }
        if (is_int) {
            const long long s0 = (long long)a, e0 = (long long)b, d = (long long)st;
            if (d <= 0) {
                err = "Step must be > 0.";
                return false;
            }
            for (long long x = s0, i = 0; x <= e0 && i < 100000; x += d, ++i) out.push_back((double)x);
        } else {
            for (int i = 0; i < 10000; ++i) {
                const double x = a + st * i;
                if (x > b + 1e-12) break;
                out.push_back(x);
            }
        }
        if (out.empty()) out.push_back(a);
        return true;
    }
    if (const Json *l = v.get("list")) {
        if (l->kind != Json::Array || l->arr.empty()) {
            err = "List is empty.";
            return false;
        }
        for (const auto &x : l->arr) {
            if (x.kind != Json::Number || !std::isfinite(x.num)) {
                err = "Invalid number in list";
                return false;
            }
            out.push_back(is_int ? (double)(long long)x.num : x.num);
        }
        return true;
    }
    err = "expected {\"range\": [...]} or {\"list\": [...]}";
    return false;
}

inline std::string run_dir(const std::string &root, int idx, int total) {
    if (total <= 1) return root;
    char b[16];
    snprintf(b, sizeof(b), "run_%04d", idx);
    return root.empty() ? std::string(b) : root + "/" + b;
}

// Parse a batch file's text into the expanded runs (model defaults from the CLI).
inline bool parse_sweep(const std::string &text, SweepSpec &sp, std::string &err) {
    Json j;
    Parser p(text);
    if (!p.parse(j, err)) return false;
    if (j.kind != Json::Object) {
        err = "the batch file must hold a JSON object";
        return false;
    }
    if (const Json *m = j.get("model")) sp.model = m->str;
    if (sp.model != "misfit" && sp.model != "cvd" && sp.model != "elastic") {
        err = "model must be misfit, cvd or elastic";
        return false;
    }
    const Json *od = j.get("out_dir");
    if (!od || od->kind != Json::String || od->str.empty()) {
        err = "out_dir is required";
        return false;
    }
    sp.out_dir = od->str;
    if (const Json *g = j.get("grid")) {
        if (g->kind != Json::Array || g->arr.size() != 3) {
            err = "grid needs [L, M, N]";
            return false;
        }
        sp.L = (int)g->arr[0].num;
        sp.M = (int)g->arr[1].num;
        sp.N = (int)g->arr[2].num;
    }
    if (const Json *x = j.get("input_dir")) sp.input_dir = x->str;
    if (const Json *x = j.get("hbm_budget_gb")) sp.budget_gb = x->num;
    if (const Json *x = j.get("max_active")) sp.max_active = (int)x->num;
    // defaults of the model's CLI (MIS:125-143, CVD:33-53, ELA defaults)
    RunSpec base{};
    const bool cvd = sp.model == "cvd", ela = sp.model == "elastic";
    base.u0 = cvd ? 0.01 : 0.05;
    base.con0 = 0.2;
    base.sig = cvd ? 0.03 : 0.05;
    base.dt = ela ? 0.1 : 0.05;
    base.dx = 0.125;
    base.steps = cvd ? 2000 : (ela ? 2002 : 200);
    base.mod = cvd || ela ? 200 : 25;
    base.seed = 20200604u;
    base.benchel = 1.7;
    static const char *order[] = {"u0", "con0", "sig", "dt", "dx", "steps", "mod", "seed", "benchel"};
    static const bool is_int[] = {false, false, false, false, false, true, true, true, false};
    std::vector<std::pair<int, std::vector<double>>> axes;
    const Json *params = j.get("params");
    if (params && params->kind != Json::Object) {
        err = "params must be an object";
        return false;
    }
    if (params)
        for (const auto &kv : params->obj) {
            int which = -1;
            for (int k = 0; k < 9; ++k)
                if (kv.first == order[k]) which = k;
            if (which < 0) {
                err = "unknown parameter " + kv.first;
                return false;
            }
        }
    long long total = 1;
    for (int k = 0; k < 9; ++k) {
        const Json *v = params ? params->get(order[k]) : nullptr;
        if (!v) continue;
        std::vector<double> vals;
        if (!param_values(*v, is_int[k], vals, err)) {
            err = std::string(order[k]) + ": " + err;
            return false;
        }
        if (total > 5000 / (long long)vals.size()) {
            err = "Too many runs (> 5000). Reduce ranges/lists (limit: 5000).";
            return false;
        }
        total *= (long long)vals.size();
        axes.emplace_back(k, std::move(vals));
    }
    std::vector<size_t> idx(axes.size(), 0);
    for (long long i = 0; i < total; ++i) {
        RunSpec r = base;
        for (size_t a = 0; a < axes.size(); ++a) {
            const double v = axes[a].second[idx[a]];
            switch (axes[a].first) {
                case 0: r.u0 = v; break;
                case 1: r.con0 = v; break;
                case 2: r.sig = v; break;
                case 3: r.dt = v; break;
                case 4: r.dx = v; break;
                case 5: r.steps = (int)v; break;
                case 6: r.mod = (int)v; break;
                case 7: r.seed = (unsigned)(long long)v; break;
                default: r.benchel = v; break;
            }
        }
        r.index = (int)i + 1;
        r.total = (int)total;
        r.out_dir = run_dir(sp.out_dir, r.index, r.total);
        sp.runs.push_back(r);
        for (int a = (int)axes.size() - 1; a >= 0; --a) {  // odometer, last parameter fastest
            if (++idx[a] < axes[a].second.size()) break;
            idx[a] = 0;
        }
    }
    return true;
}

// Shortest decimal that reads back as v (the form Qt's JSON writer uses for doubles).
inline std::string json_number(double v) {
    if (v == std::floor(v) && std::fabs(v) < 1e15) {
        char b[32];
        snprintf(b, sizeof(b), "%.0f", v);
        return b;
    }
    char b[64];
    auto res = std::to_chars(b, b + sizeof(b), v);
    return std::string(b, res.ptr);
}

// params.json of one run, with the GUI's keys (MainWindow.cpp:2430-2471) in the sorted
// order and four-space indentation of QJsonDocument::Indented.
inline std::string params_json(const SweepSpec &sp, const RunSpec &r) {
    std::string s = "{\n";
    s += "    \"mode\": \"experiment\",\n";
    s += "    \"out_dir\": \"" + r.out_dir + "\",\n";
    s += "    \"params\": {\n";
    std::vector<std::pair<std::string, std::string>> p;
    if (sp.model == "elastic") {
        p.emplace_back("benchel", json_number(r.benchel));
        if (!sp.input_dir.empty()) p.emplace_back("input_dir", "\"" + sp.input_dir + "\"");
    }
    p.emplace_back("con0", json_number(r.con0));
    p.emplace_back("dt", json_number(r.dt));
    p.emplace_back("dx", json_number(r.dx));
    p.emplace_back("mod", std::to_string(r.mod));
    p.emplace_back("model", "\"" + sp.model + "\"");
    p.emplace_back("seed", std::to_string(r.seed));
    p.emplace_back("sig", json_number(r.sig));
    p.emplace_back("steps", std::to_string(r.steps));
    p.emplace_back("u0", json_number(r.u0));
    for (size_t i = 0; i < p.size(); ++i)
        s += "        \"" + p[i].first + "\": " + p[i].second + (i + 1 < p.size() ? ",\n" : "\n");
    s += "    },\n";
    s += "    \"run_index\": " + std::to_string(r.index) + ",\n";
    s += "    \"run_total\": " + std::to_string(r.total) + "\n";
    s += "}\n";
    return s;
}

}  // namespace sweep
}  // namespace pfc

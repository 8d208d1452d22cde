// Histogram / Accum / score (src/stats.hpp:10-83), PSNR (src/main.cpp:272-277) and the JSON object of a segment
// (src/main.cpp:727-757), in the same arithmetic so that outputs diff cleanly against the reference's.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/es_b200.h"

namespace {
constexpr double kLo = -500.0, kStep = 0.05;

double clamp100(double v) { return std::min(std::max(v, 0.0), 100.0); }
double kept(double d, double r) { return r > 0 ? 100.0 * std::sqrt(d / r) : NAN; }

std::string num(double v, int digits)
{
    if (!std::isfinite(v)) return "null";
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.*f", digits, v);
    return buf;
}

std::string list(std::initializer_list<double> vs, int digits)
{
    std::string out = "[";
    for (double v : vs) out += (out.size() > 1 ? ", " : "") + num(v, digits);
    return out + "]";
}
}  // namespace

extern "C" {

void es_histogram_add(es_histogram *hist, double pct)
{
    const int b = (int)std::lround((std::clamp(pct, kLo, -kLo) - kLo) / kStep);
    hist->bins[b]++;
    hist->n++;
}

double es_histogram_quantile(const es_histogram *hist, double q)
{
    if (!hist->n) return NAN;
    const double target = q * (double)(hist->n - 1);
    uint64_t seen = 0;
    for (int b = 0; b < ES_HIST_BINS; b++) {
        seen += hist->bins[b];
        if ((double)seen > target) return kLo + (double)b * kStep;
    }
    return -kLo;
}

void es_accum_init(es_accum *a)
{
    std::memset(a, 0, sizeof *a);
    a->vmaf_min = 1e9;
}

void es_accum_merge(es_accum *a, const es_accum *o)
{
    a->frames += o->frames;
    a->vmaf += o->vmaf;
    a->vmaf_min = std::min(a->vmaf_min, o->vmaf_min);
    a->cambi += o->cambi;
    a->cambi_source += o->cambi_source;
    a->own += o->own;
    a->mine += o->mine;
    for (int i = 0; i < 3; i++) {
        a->psnr[i] += o->psnr[i];
        a->color_r[i] += o->color_r[i];
        a->color_d[i] += o->color_d[i];
        a->all_r[i] += o->all_r[i];
        a->all_d[i] += o->all_d[i];
        a->st_r[i] += o->st_r[i];
        a->st_d[i] += o->st_d[i];
        for (int b = 0; b < ES_HIST_BINS; b++) a->amount[i].bins[b] += o->amount[i].bins[b];
        a->amount[i].n += o->amount[i].n;
    }
    for (int i = 0; i < 2; i++) {
        a->sh_all_r[i] += o->sh_all_r[i];
        a->sh_all_x[i] += o->sh_all_x[i];
        a->sh_st_r[i] += o->sh_st_r[i];
        a->sh_st_x[i] += o->sh_st_x[i];
        for (int b = 0; b < ES_HIST_BINS; b++) a->matching[i].bins[b] += o->matching[i].bins[b];
        a->matching[i].n += o->matching[i].n;
    }
    for (int b = 0; b < ES_HIST_BINS; b++) a->lasting.bins[b] += o->lasting.bins[b];
    a->lasting.n += o->lasting.n;
}

void es_accum_score(const es_accum *a, const es_weights *weights, es_parts *out)
{
    const es_weights w = weights ? *weights : es_weights{0.30, 0.30, 0.25, 0.15};
    es_parts p;
    p.fidelity = clamp100(a->vmaf / (double)a->frames);
    p.texture = a->lasting.n >= 100 ? clamp100(es_histogram_quantile(&a->lasting, 0.5)) / 2 + clamp100(es_histogram_quantile(&a->lasting, 0.1)) / 2
                                    : NAN;
    p.banding = clamp100(100.0 * (1 - (a->cambi - a->cambi_source) / (double)a->frames / 5.0));
    p.grain = clamp100(100.0 - std::fabs(kept(a->all_d[0], a->all_r[0]) - 100.0));
    double total = 0, weight = 0;
    const double v[4] = {p.fidelity, p.texture, p.banding, p.grain}, k[4] = {w.fidelity, w.texture, w.banding, w.grain};
    for (int i = 0; i < 4; i++)
        if (!std::isnan(v[i])) {
            total += v[i] * k[i];
            weight += k[i];
        }
    p.score = total / weight;
    *out = p;
}

size_t es_accum_json(const es_accum *a, char *buf, size_t size)
{
    es_parts p;
    es_accum_score(a, nullptr, &p);
    const double f = (double)a->frames;
    auto q = [](const es_histogram &h, double x) { return es_histogram_quantile(&h, x); };
    const std::string out =
        "{\"frames\": " + std::to_string(a->frames) + ", \"score\": " + num(p.score, 4) + ", \"fidelity\": " + num(p.fidelity, 4) +
        ", \"texture\": " + num(p.texture, 4) + ", \"banding\": " + num(p.banding, 4) + ", \"grain\": " + num(p.grain, 4) +
        ", \"vmaf\": " + num(a->vmaf / f, 6) + ", \"vmaf_min\": " + num(a->vmaf_min, 6) +
        ", \"psnr_y\": " + num(a->psnr[0] / f, 4) + ", \"psnr_cb\": " + num(a->psnr[1] / f, 4) + ", \"psnr_cr\": " + num(a->psnr[2] / f, 4) +
        ", \"cambi\": " + num(a->cambi / f, 6) + ", \"cambi_source\": " + num(a->cambi_source / f, 6) +
        ", \"lasting\": {\"windows\": " + std::to_string(a->lasting.n) + ", \"median\": " + num(q(a->lasting, 0.5), 3) +
        ", \"worst_tenth\": " + num(q(a->lasting, 0.1), 3) + ", \"total\": " + num(a->own > 0 ? 100.0 * a->mine / a->own : NAN, 3) + "}" +
        ", \"amount\": {\"all\": " + list({kept(a->all_d[0], a->all_r[0]), kept(a->all_d[1], a->all_r[1]), kept(a->all_d[2], a->all_r[2])}, 3) +
        ", \"structure\": " + list({kept(a->st_d[0], a->st_r[0]), kept(a->st_d[1], a->st_r[1]), kept(a->st_d[2], a->st_r[2])}, 3) +
        ", \"median\": " + list({q(a->amount[0], 0.5), q(a->amount[1], 0.5), q(a->amount[2], 0.5)}, 3) +
        ", \"worst_tenth\": " + list({q(a->amount[0], 0.1), q(a->amount[1], 0.1), q(a->amount[2], 0.1)}, 3) + "}" +
        ", \"matching\": {\"all\": " + list({100.0 * a->sh_all_x[0] / a->sh_all_r[0], 100.0 * a->sh_all_x[1] / a->sh_all_r[1]}, 3) +
        ", \"structure\": " + list({100.0 * a->sh_st_x[0] / a->sh_st_r[0], 100.0 * a->sh_st_x[1] / a->sh_st_r[1]}, 3) +
        ", \"median\": " + list({q(a->matching[0], 0.5), q(a->matching[1], 0.5)}, 3) +
        ", \"worst_tenth\": " + list({q(a->matching[0], 0.1), q(a->matching[1], 0.1)}, 3) + "}" +
        ", \"color_source\": " + list({a->color_r[0] / f, a->color_r[1] / f, a->color_r[2] / f}, 4) +
        ", \"color_encode\": " + list({a->color_d[0] / f, a->color_d[1] / f, a->color_d[2] / f}, 4) + "}";
    if (buf && size) {
        const size_t n = std::min(out.size(), size - 1);
        std::memcpy(buf, out.data(), n);
        buf[n] = '\0';
    }
    return out.size();
}

double es_psnr(uint64_t sse, uint64_t n, int depth)
{
    const double mse = (double)sse / (double)n, peak = (double)((1 << depth) - 1);
    return std::min(10.0 * std::log10(peak * peak / std::max(mse, 1e-16)), 6.0 * depth + 12);
}

size_t es_per_frame_json(const double *vmaf, const double *cambi, const double *cambi_source, const double *psnr_y, long n,
                         char *buf, size_t size)
{
    // src/main.cpp:767-774: {"vmaf": [...], "cambi": [...], "cambi_source": [...], "psnr_y": [...]}, 6 digits (3 for
    // PSNR), comma-separated without spaces; without VMAF figures, "vmaf": null
    std::string out = "{\"vmaf\": ";
    auto arr = [&](const double *v, int digits) {
        std::string s = "[";
        char tmp[64];
        for (long i = 0; i < n; i++) {
            std::snprintf(tmp, sizeof tmp, "%s%.*f", i ? "," : "", digits, v[i]);
            s += tmp;
        }
        return s + "]";
    };
    out += vmaf ? arr(vmaf, 6) : std::string("null");
    out += ", \"cambi\": " + arr(cambi, 6) + ", \"cambi_source\": " + arr(cambi_source, 6) + ", \"psnr_y\": " + arr(psnr_y, 3) + "}";
    if (buf && size) {
        const size_t k = std::min(size - 1, out.size());
        std::memcpy(buf, out.data(), k);
        buf[k] = '\0';
    }
    return out.size();
}

}  // extern "C"

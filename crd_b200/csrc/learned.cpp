// The learned cost model (learned.hpp).

#include "learned.hpp"

#include "kernels.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <sstream>
#include <vector>

namespace crdfft
{
namespace
{

float lg2(double v) { return v > 0.0 ? static_cast<float>(std::log2(v)) : -1.0f; }

struct Model
{
    int in_dim = 0;
    int hidden = 0;
    std::vector<float> mean, stdev; // feature normalisation
    float t_mean = 0.0f, t_std = 1.0f; // target normalisation: log(ms) = t_mean + t_std * output
    std::vector<float> params;      // [W1 H x D][b1 H][W2 H x H][b2 H][W3 H][b3]
};

// Two models: slot 0 ranks a pass's launch shapes ("crdfft-mlp 1"), slot 1 a transform's decompositions
// ("crdfft-mlp-decomp 1").
std::mutex g_mu;
Model g_models[2];
bool g_ready[2] = {false, false};
const char* const kTags[2] = {"crdfft-mlp", "crdfft-mlp-decomp"};

size_t param_count(int d, int h) { return static_cast<size_t>(h) * d + h + static_cast<size_t>(h) * h + h + h + 1; }

} // namespace

// Features of a pass under a launch shape, all O(1) in magnitude:
//   0 log2 n              1 stages                   2-8 stages of radix 16, 8, 4, 2, 3, 5, 7
//   9 log2 lines          10 log2 lines a group      11 column map            12 direct load   13 direct store
//   14 conjugation/scale  15 four-step twiddle       16-17 unit element stride in / out
//   18-19 log2 element stride in / out               20-21 unit line distance in / out
//   22 padded layout (a line or group distance that is not a multiple of 16 elements)
//   23 pipelined kernel   24 32 points a thread      25 log2 lines a CTA      26 log2 threads a CTA
//   27 shared memory / 64 KiB                        28 log2 bytes moved      29 log2 CTAs
//   30 a compile-time schedule exists                31 1 (bias feature, constant)
void pass_features(const PassDesc& d, const PassShape& sh, float* f)
{
    for (int i = 0; i < kPassFeatures; ++i)
        f[i] = 0.0f;
    f[0] = lg2(d.n);
    f[1] = static_cast<float>(d.nstages);
    for (int s = 0; s < d.nstages; ++s)
    {
        switch (d.radix[s])
        {
            case 16: f[2] += 1; break;
            case 8: f[3] += 1; break;
            case 4: f[4] += 1; break;
            case 2: f[5] += 1; break;
            case 3: f[6] += 1; break;
            case 9: f[6] += 2; break;
            case 25: f[7] += 2; break;
            case 5: f[7] += 1; break;
            case 7: f[8] += 1; break;
            default: break;
        }
    }
    f[9] = lg2(static_cast<double>(d.lines));
    f[10] = lg2(static_cast<double>(d.lines_per_group));
    f[11] = sh.map == PassMap::Col ? 1.0f : 0.0f;
    f[12] = sh.direct_load ? 1.0f : 0.0f;
    f[13] = sh.direct_store ? 1.0f : 0.0f;
    f[14] = (d.conj_in || d.conj_out || d.scale != 1.0f) ? 1.0f : 0.0f;
    f[15] = d.ftw_M != 0 ? 1.0f : 0.0f;
    f[16] = d.in.estride == 1 ? 1.0f : 0.0f;
    f[17] = d.out.estride == 1 ? 1.0f : 0.0f;
    f[18] = lg2(static_cast<double>(d.in.estride));
    f[19] = lg2(static_cast<double>(d.out.estride));
    f[20] = d.in.ldist == 1 ? 1.0f : 0.0f;
    f[21] = d.out.ldist == 1 ? 1.0f : 0.0f;
    auto padded = [](const LineMap& m) {
        return (m.ldist != 1 && m.ldist % 16 != 0) || (m.gdist % 16 != 0 && m.gdist != 0);
    };
    f[22] = (padded(d.in) || padded(d.out)) ? 1.0f : 0.0f;
    f[23] = sh.pipelined ? 1.0f : (sh.tma_store ? 0.5f : 0.0f); // bulk-copy-fed, tensor-store row pass, classic
    f[24] = sh.points_per_thread == 32 ? 1.0f : (sh.wide_regs ? 0.5f : 0.0f); // 16 narrow, 16 wide, 32
    f[25] = lg2(sh.lines_per_cta);
    f[26] = lg2(static_cast<double>(sh.threads_per_line) * sh.lines_per_cta);
    f[27] = static_cast<float>(sh.smem_bytes) / 65536.0f;
    f[28] = lg2(16.0 * d.n * static_cast<double>(d.lines));
    f[29] = lg2(static_cast<double>((d.lines + sh.lines_per_cta - 1) / sh.lines_per_cta));
    f[30] = pass_has_static(d, sh.points_per_thread) ? 1.0f : 0.0f;
    f[31] = 1.0f;
}

namespace
{

// Parses one model from `in` (its tag already read); 0 or -1.
int parse_model(std::istream& in, Model* out)
{
    int version = 0;
    if (!(in >> version) || version != 1)
        return -1;
    Model m;
    std::string w;
    if (!(in >> w >> m.in_dim >> m.hidden) || w != "dims" || m.in_dim != kPassFeatures || m.hidden < 1 ||
        m.hidden > 1024)
        return -1;
    m.mean.resize(m.in_dim);
    m.stdev.resize(m.in_dim);
    if (!(in >> w) || w != "mean")
        return -1;
    for (float& v : m.mean)
        if (!(in >> v))
            return -1;
    if (!(in >> w) || w != "std")
        return -1;
    for (float& v : m.stdev)
        if (!(in >> v) || !(v > 0.0f))
            return -1;
    if (!(in >> w >> m.t_mean >> m.t_std) || w != "target" || !(m.t_std > 0.0f))
        return -1;
    size_t count = 0;
    if (!(in >> w >> count) || w != "params" || count != param_count(m.in_dim, m.hidden))
        return -1;
    m.params.resize(count);
    for (float& v : m.params)
        if (!(in >> v) || !std::isfinite(v))
            return -1;
    *out = std::move(m);
    return 0;
}

std::string export_model(int slot)
{
    const Model& m = g_models[slot];
    std::ostringstream o;
    char buf[32];
    auto put = [&](float v) {
        std::snprintf(buf, sizeof(buf), " %.9g", static_cast<double>(v));
        o << buf;
    };
    o << kTags[slot] << " 1\ndims " << m.in_dim << ' ' << m.hidden << "\nmean";
    for (float v : m.mean)
        put(v);
    o << "\nstd";
    for (float v : m.stdev)
        put(v);
    o << "\ntarget";
    put(m.t_mean);
    put(m.t_std);
    o << "\nparams " << m.params.size() << '\n';
    for (size_t i = 0; i < m.params.size(); ++i)
    {
        put(m.params[i]);
        if (i % 8 == 7)
            o << '\n';
    }
    o << '\n';
    return o.str();
}

// The forward pass of the same network the device kernels train (mlp.cu), on the host: normalise, two ReLU layers,
// one linear output, de-normalise.
float predict_model(const Model& m, const float* feat)
{
    const int D = m.in_dim, H = m.hidden;
    const float* W1 = m.params.data();
    const float* b1 = W1 + static_cast<size_t>(H) * D;
    const float* W2 = b1 + H;
    const float* b2 = W2 + static_cast<size_t>(H) * H;
    const float* W3 = b2 + H;
    const float b3 = W3[H];
    std::vector<float> x(D), a1(H), a2(H);
    for (int k = 0; k < D; ++k)
        x[k] = (feat[k] - m.mean[k]) / m.stdev[k];
    for (int o = 0; o < H; ++o)
    {
        float s = b1[o];
        for (int k = 0; k < D; ++k)
            s += W1[static_cast<size_t>(o) * D + k] * x[k];
        a1[o] = s > 0.0f ? s : 0.0f;
    }
    for (int o = 0; o < H; ++o)
    {
        float s = b2[o];
        for (int k = 0; k < H; ++k)
            s += W2[static_cast<size_t>(o) * H + k] * a1[k];
        a2[o] = s > 0.0f ? s : 0.0f;
    }
    float y = b3;
    for (int k = 0; k < H; ++k)
        y += W3[k] * a2[k];
    return m.t_mean + m.t_std * y;
}

} // namespace

// A model text holds one or both models, each introduced by its tag; every model in it must parse, or nothing is
// imported. A model replaces the one in its slot; the other slot is kept.
int learned_import(const std::string& text)
{
    std::istringstream in(text);
    std::string tag;
    Model got[2];
    bool have[2] = {false, false};
    while (in >> tag)
    {
        int slot = -1;
        for (int i = 0; i < 2; ++i)
            if (tag == kTags[i])
                slot = i;
        if (slot < 0 || parse_model(in, &got[slot]) != 0)
            return -1;
        have[slot] = true;
    }
    if (!have[0] && !have[1])
        return -1;
    std::lock_guard<std::mutex> lk(g_mu);
    for (int i = 0; i < 2; ++i)
        if (have[i])
        {
            g_models[i] = std::move(got[i]);
            g_ready[i] = true;
        }
    return 0;
}

std::string learned_export()
{
    std::lock_guard<std::mutex> lk(g_mu);
    std::string out;
    for (int i = 0; i < 2; ++i)
        if (g_ready[i])
            out += export_model(i);
    return out;
}

bool learned_ready()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ready[0];
}

bool learned_decomp_ready()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ready[1];
}

void learned_forget()
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int i = 0; i < 2; ++i)
    {
        g_ready[i] = false;
        g_models[i] = Model{};
    }
}

float learned_predict(const float* feat)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ready[0] ? predict_model(g_models[0], feat) : 0.0f;
}

float learned_decomp_predict(const float* feat)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ready[1] ? predict_model(g_models[1], feat) : 0.0f;
}

// Features of a 1-D decomposition choice, all O(1) in magnitude:
//   0 log2 n              1 log2 batch               2 log2 bytes of input     3-5 single pass / cluster / four-step
//   6 log2 n1 (columns)   7 log2 n2 (rows)           8 |log2 (n1 / n2)|        9-10 n1, n2 have compile-time schedules
//   11-17 stages of radix 16, 8, 4, 2, 3, 5, 7 in n1    18-24 the same for n2
//   25 n2 a multiple of 16 (whole column tiles)      26 unit strides and packed  27 padded distances
//   28 precision (0 FP32, 1 tensor-core form)        29 waves of the four-step at the default wave size (log2)
//   30 the column pass takes the tensor-copy kernel  31 1 (bias feature, constant)
void decomp_features(long long n, int kind, long long n1, long long batch, bool packed_unit, bool padded,
                     int precision, const int* r1, int s1, const int* r2, int s2, bool stat1, bool stat2,
                     bool tma_col, float* f)
{
    for (int i = 0; i < kPassFeatures; ++i)
        f[i] = 0.0f;
    const long long n2 = kind == 3 ? n / n1 : 1;
    const long long a = kind == 3 ? n1 : n;
    f[0] = lg2(static_cast<double>(n));
    f[1] = lg2(static_cast<double>(batch));
    f[2] = lg2(8.0 * static_cast<double>(n) * static_cast<double>(batch));
    f[3 + (kind == 1 ? 0 : kind == 2 ? 1 : 2)] = 1.0f;
    f[6] = lg2(static_cast<double>(a));
    f[7] = lg2(static_cast<double>(n2));
    f[8] = std::fabs(f[6] - f[7]);
    f[9] = stat1 ? 1.0f : 0.0f;
    f[10] = stat2 ? 1.0f : 0.0f;
    auto count = [&](const int* r, int s, int at) {
        for (int i = 0; i < s; ++i)
            switch (r[i])
            {
                case 16: f[at + 0] += 1; break;
                case 8: f[at + 1] += 1; break;
                case 4: f[at + 2] += 1; break;
                case 2: f[at + 3] += 1; break;
                case 3: f[at + 4] += 1; break;
                case 9: f[at + 4] += 2; break;
                case 25: f[at + 5] += 2; break;
                case 5: f[at + 5] += 1; break;
                case 7: f[at + 6] += 1; break;
                default: break;
            }
    };
    count(r1, s1, 11);
    count(r2, s2, 18);
    f[25] = (kind == 3 && n2 % 16 == 0) ? 1.0f : 0.0f;
    f[26] = packed_unit ? 1.0f : 0.0f;
    f[27] = padded ? 1.0f : 0.0f;
    f[28] = precision != 0 ? 1.0f : 0.0f;
    f[29] = kind == 3 ? lg2(std::max(1.0, 8.0 * n * static_cast<double>(batch) / static_cast<double>(512 << 20)))
                      : 0.0f;
    f[30] = tma_col ? 1.0f : 0.0f;
    f[31] = 1.0f;
}

} // namespace crdfft

// guide_oracle.cpp — f64 restatement of the learned proposal's network for
// gradient checks. TEST INFRASTRUCTURE ONLY (tests/ import it through
// oracle.py); the CUDA backend never calls it.
//
// The reference has no counterpart (path guiding is unimplemented there,
// ROADMAP.md:34), so this oracle restates the network as specified: the
// hash-grid encoding (16 levels x 2 features; 2x2x2 vertex blocks placed by
// a spatial hash with the instant-ngp primes, densely on coarse levels), a
// 48-64-64-64-48
// ReLU MLP, and the loss -w log q(wi) of an 8-lobe von Mises-Fisher
// mixture. Arithmetic is f64; the values the GPU stores in bf16 (layer
// inputs, activations and the back-propagated dZ fed to the tensor cores)
// are rounded to bf16 here too, so the two agree to accumulation order.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

const int L = 16, T_LOG2 = 19, IN = 48, HID = 64, OUT = 48, LOBES = 8;
const uint32_t T = 1u << T_LOG2;
const int NW[4] = {HID * IN, HID * HID, HID * HID, OUT * HID};
const int WOFF[4] = {0, HID * IN, HID * IN + HID * HID, HID * IN + 2 * HID * HID};
const int NWEIGHTS = HID * IN + 2 * HID * HID + OUT * HID;
const int LIN[4] = {IN, HID, HID, HID}, LOUT[4] = {HID, HID, HID, OUT};

double bf16(double x) {
    // round-to-nearest-even to bfloat16 via the f32 bit pattern
    float f = (float)x;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7F800000u) == 0x7F800000u) return f;
    uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    r &= 0xFFFF0000u;
    memcpy(&f, &r, 4);
    return f;
}

double half_to_double(uint16_t h) {
    uint32_t s = (h >> 15) & 1u, e = (h >> 10) & 31u, m = h & 1023u;
    double v;
    if (e == 0) v = std::ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = std::ldexp((double)(m | 1024u), (int)e - 25);
    return s ? -v : v;
}

uint32_t grid_index(uint32_t x, uint32_t y, uint32_t z, uint32_t res1, bool dense) {
    // 2x2x2 vertex blocks of 8 consecutive entries; blocks placed densely or by
    // the Teschner et al. spatial hash (as render.rs_b200/csrc/guide.cuh)
    const uint32_t intra = (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
    const uint32_t bx = x >> 1, by = y >> 1, bz = z >> 1, nb = (res1 + 1u) >> 1;
    const uint32_t block = dense ? bx + (by + bz * nb) * nb : (bx * 1u ^ by * 2654435761u ^ bz * 805459861u);
    return (block * 8u + intra) & (T - 1u);
}

struct Corner {
    uint32_t idx[L][8];
    double w[L][8];
};

void encode(const double* table, const float* res, const float* lo, const float* inv_ext, const float* p, double* feat,
            Corner* cr) {
    double pn[3];
    for (int a = 0; a < 3; a++) {
        float q = (p[a] - lo[a]) * inv_ext[a];  // f32 like the GPU
        pn[a] = std::fmin(std::fmax((double)q, 0.0), 1.0);
    }
    for (int l = 0; l < L; l++) {
        float r = res[l];
        uint32_t res1 = (uint32_t)r + 2u;
        const uint64_t nb = (res1 + 1u) >> 1;
        bool dense = nb * nb * nb * 8u <= T;
        float fx = (float)pn[0] * r, fy = (float)pn[1] * r, fz = (float)pn[2] * r;
        float ix = std::floor(fx), iy = std::floor(fy), iz = std::floor(fz);
        double tx = fx - ix, ty = fy - iy, tz = fz - iz;
        uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
        double a0 = 0, a1 = 0;
        for (int c = 0; c < 8; c++) {
            uint32_t dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
            double w = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
            uint32_t id = grid_index(x0 + dx, y0 + dy, z0 + dz, res1, dense);
            a0 += w * table[((size_t)l * T + id) * 2];
            a1 += w * table[((size_t)l * T + id) * 2 + 1];
            cr->idx[l][c] = id;
            cr->w[l][c] = w;
        }
        feat[2 * l] = a0;
        feat[2 * l + 1] = a1;
    }
}

// -w log q(wi) and its gradient with respect to the raw outputs.
double mixture_loss_grad(const double* o, const double* wi, double weight, double* g) {
    double mx = -1e300;
    for (int j = 0; j < LOBES; j++) mx = std::fmax(mx, o[5 * j + 4]);
    double pi[LOBES], lv[LOBES], kap[LOBES], len[LOBES], dmw[LOBES], mu[LOBES][3], sw = 0;
    for (int j = 0; j < LOBES; j++) {
        double v[3] = {o[5 * j], o[5 * j + 1], o[5 * j + 2]};
        len[j] = std::fmax(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 1e-8);
        for (int a = 0; a < 3; a++) mu[j][a] = v[a] / len[j];
        kap[j] = std::exp(std::fmin(std::fmax(o[5 * j + 3], -4.0), 9.0));
        pi[j] = std::exp(o[5 * j + 4] - mx);
        sw += pi[j];
        dmw[j] = mu[j][0] * wi[0] + mu[j][1] * wi[1] + mu[j][2] * wi[2];
    }
    double lmax = -1e300;
    for (int j = 0; j < LOBES; j++) {
        pi[j] /= sw;
        double k = kap[j];
        double norm = std::log(k) - std::log(2 * M_PI) - std::log1p(-std::exp(-2 * k));
        lv[j] = std::log(std::fmax(pi[j], 1e-30)) + norm + k * (dmw[j] - 1);
        lmax = std::fmax(lmax, lv[j]);
    }
    double s = 0;
    for (int j = 0; j < LOBES; j++) s += std::exp(lv[j] - lmax);
    double logq = lmax + std::log(s);
    for (int j = 0; j < LOBES; j++) {
        double r = std::exp(lv[j] - logq), k = kap[j];
        double dlk = 1 / k + (dmw[j] - 1) - 2 / std::fmax(std::exp(2 * k) - 1, 1e-30);
        double lk = o[5 * j + 3];
        g[5 * j + 3] = (lk > -4 && lk < 9) ? -weight * r * dlk * k : 0;
        for (int a = 0; a < 3; a++) g[5 * j + a] = (wi[a] - mu[j][a] * dmw[j]) * (-weight * r * k / len[j]);
        g[5 * j + 4] = -weight * (r - pi[j]);
    }
    for (int j = 5 * LOBES; j < OUT; j++) g[j] = 0;
    return -weight * logq;
}

}  // namespace

extern "C" {

// mlp: f32 params (weights row-major [out][in] per layer, then biases);
// table: fp16 bit patterns, levels * 2^19 * 2. Outputs (all optional):
// raw n*48, g_mlp (params), g_table (levels*2^19*2), loss (sum).
int oracle_guide_eval(const float* mlp, const uint16_t* table16, const float* res, const float* lo,
                      const float* inv_ext, const float* rec, uint32_t n, double* raw, double* g_mlp, float* g_table,
                      double* loss) {
    std::vector<double> table((size_t)L * T * 2);
    for (size_t i = 0; i < table.size(); i++) table[i] = half_to_double(table16[i]);
    std::vector<double> W(NWEIGHTS);
    for (int i = 0; i < NWEIGHTS; i++) W[i] = bf16(mlp[i]);
    const float* B = mlp + NWEIGHTS;
    if (g_mlp) memset(g_mlp, 0, sizeof(double) * (NWEIGHTS + 3 * HID + OUT));
    if (g_table) memset(g_table, 0, sizeof(float) * table.size());
    double total = 0;
    for (uint32_t s = 0; s < n; s++) {
        const float* r = rec + 16 * (size_t)s;
        Corner cr;
        double x[4][HID];  // layer inputs (bf16-rounded), x[0] has IN entries
        double feat[IN] = {0};
        encode(table.data(), res, lo, inv_ext, r, feat, &cr);
        for (int k = 0; k < 6; k++) feat[32 + k] = r[3 + k];
        for (int k = 0; k < IN; k++) x[0][k] = bf16(feat[k]);
        double out[OUT];
        for (int l = 0; l < 4; l++) {
            for (int o = 0; o < LOUT[l]; o++) {
                double z = 0;
                for (int k = 0; k < LIN[l]; k++) z += W[WOFF[l] + o * LIN[l] + k] * x[l][k];
                z += (double)(float)((double)0 + B[l * HID + o]);
                if (l < 3) x[l + 1][o] = bf16(std::fmax((float)z, 0.0f));
                else out[o] = z;
            }
        }
        if (raw)
            for (int o = 0; o < OUT; o++) raw[(size_t)s * OUT + o] = out[o];
        double wi[3] = {r[9], r[10], r[11]};
        double dz[HID];
        total += mixture_loss_grad(out, wi, r[12], dz);
        if (!g_mlp && !g_table) continue;
        for (int l = 3; l >= 0; l--) {
            double dzr[HID];
            for (int o = 0; o < LOUT[l]; o++) {
                dzr[o] = bf16(dz[o]);
                if (g_mlp) g_mlp[NWEIGHTS + l * HID + o] += (float)dz[o];
            }
            if (g_mlp)
                for (int o = 0; o < LOUT[l]; o++)
                    for (int k = 0; k < LIN[l]; k++) g_mlp[WOFF[l] + o * LIN[l] + k] += dzr[o] * x[l][k];
            double dh[HID];
            for (int k = 0; k < LIN[l]; k++) {
                double a = 0;
                for (int o = 0; o < LOUT[l]; o++) a += dzr[o] * W[WOFF[l] + o * LIN[l] + k];
                dh[k] = a;
            }
            if (l > 0) {
                for (int k = 0; k < HID; k++) dz[k] = x[l][k] > 0 ? (double)(float)dh[k] : 0.0;
            } else if (g_table) {
                for (int lv = 0; lv < L; lv++)
                    for (int c = 0; c < 8; c++)
                        for (int f = 0; f < 2; f++)
                            g_table[((size_t)lv * T + cr.idx[lv][c]) * 2 + f] +=
                                (float)(cr.w[lv][c] * (double)(float)dh[2 * lv + f]);
            }
        }
    }
    if (loss) *loss = total;
    return 0;
}

}  // extern "C"

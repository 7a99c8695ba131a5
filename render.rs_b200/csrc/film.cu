// film.cu — the AOV film and its denoiser on the device.
//
// Film: beauty, diffuse, specular, albedo, normal, depth, id + coverage per
// pixel (18 floats, RT_FILM_* in rt_cuda.h), decoded from the session's f64
// accumulator and its 12-float AOV sums as render_pt_film does
// (src/raytracer/metal/renderer.rs:180-217), with each pixel's own sample
// count in place of the frame's spp (they agree unless adaptive sampling
// stopped a pixel early).
//
// Denoiser: the reference's edge-avoiding a-trous wavelet filter
// (src/output/denoise.rs:28-139, after Dammertz et al. 2010): the diffuse
// layer is divided by max(albedo, 0.05), filtered in 5 passes of a 5x5
// B3-spline kernel with holes 1, 2, 4, 8, 16, each tap weighted by
// exp(-dlum^2 / sigma^2) (sigma 8, halved per pass), max(n.n0, 0)^32,
// exp(-(dz / median depth)^2 / 0.02) and zero across object ids, then
// multiplied back and the specular layer added. One thread per pixel per
// pass; the guides (normal + depth, id) are packed into planar arrays so a
// tap reads 16 + 16 + 4 bytes from L1/L2.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include "devmem.h"
#include "rt_cuda.h"

namespace rt {

std::string& accum_error();

namespace {

constexpr int FB = 256;

__global__ void k_film_decode(const double* __restrict__ accum, const float* __restrict__ aux, uint32_t npix,
                              float* __restrict__ film) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const double4 a = reinterpret_cast<const double4*>(accum)[i];
    const float* x = aux + 12ull * i;
    const double spp = a.w > 0.0 ? a.w : 1.0;
    const float inv = (float)(1.0 / spp);
    float* f = film + (size_t)RT_FILM_FLOATS * i;
    const float b[3] = {(float)(a.x / spp), (float)(a.y / spp), (float)(a.z / spp)};
    const float hits = x[11];
    for (int c = 0; c < 3; c++) {
        f[RT_FILM_BEAUTY + c] = b[c];
        f[RT_FILM_DIFFUSE + c] = x[8 + c] * inv;
        f[RT_FILM_SPECULAR + c] = fmaxf(b[c] - x[8 + c] * inv, 0.0f);
        f[RT_FILM_ALBEDO + c] = x[c] * inv;
        f[RT_FILM_NORMAL + c] = x[3 + c] * inv;
    }
    f[RT_FILM_DEPTH] = hits > 0.0f ? x[6] / fmaxf(hits, 1.0f) : 0.0f;
    f[RT_FILM_ID] = x[7];
    f[RT_FILM_ID + 1] = fminf(hits * inv, 1.0f);
}

__device__ __forceinline__ float lum3(float4 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

__global__ void k_denoise_prep(const float* __restrict__ film, uint32_t npix, float4* __restrict__ illum,
                               float4* __restrict__ guide, float* __restrict__ id) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float* f = film + (size_t)RT_FILM_FLOATS * i;
    illum[i] = make_float4(f[RT_FILM_DIFFUSE] / fmaxf(f[RT_FILM_ALBEDO], 5e-2f),
                           f[RT_FILM_DIFFUSE + 1] / fmaxf(f[RT_FILM_ALBEDO + 1], 5e-2f),
                           f[RT_FILM_DIFFUSE + 2] / fmaxf(f[RT_FILM_ALBEDO + 2], 5e-2f), 0.0f);
    guide[i] = make_float4(f[RT_FILM_NORMAL], f[RT_FILM_NORMAL + 1], f[RT_FILM_NORMAL + 2], f[RT_FILM_DEPTH]);
    id[i] = f[RT_FILM_ID];
}

__global__ void k_atrous(const float4* __restrict__ src, const float4* __restrict__ guide, const float* __restrict__ id,
                         uint32_t w, uint32_t h, int step, float inv_sigma2, float inv_depth_scale,
                         float4* __restrict__ dst) {
    const uint32_t x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (x >= w || y >= h) return;
    const float K[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    const size_t i0 = (size_t)y * w + x;
    const float4 c0 = src[i0], g0 = guide[i0];
    const float id0 = id[i0];
    float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
    float wsum = 0.0f;
    for (int kj = 0; kj < 5; kj++) {
        const int yy = (int)y + (kj - 2) * step;
        if (yy < 0 || yy >= (int)h) continue;
        for (int ki = 0; ki < 5; ki++) {
            const int xx = (int)x + (ki - 2) * step;
            if (xx < 0 || xx >= (int)w) continue;
            const size_t j = (size_t)yy * w + xx;
            const float4 c = src[j], g = guide[j];
            float wt = K[kj] * K[ki];
            const float dc = lum3(make_float4(c.x - c0.x, c.y - c0.y, c.z - c0.z, 0.f));
            wt *= __expf(-(dc * dc) * inv_sigma2);
            float nd = fmaxf(g.x * g0.x + g.y * g0.y + g.z * g0.z, 0.0f);
            nd *= nd;
            nd *= nd;
            nd *= nd;
            nd *= nd;
            nd *= nd;  // ^32
            wt *= nd;
            const float dd = (g.w - g0.w) * inv_depth_scale;
            wt *= __expf(-(dd * dd) * 50.0f);  // / 0.02
            if (fabsf(id[j] - id0) > 0.5f) wt = 0.0f;
            sum.x += c.x * wt;
            sum.y += c.y * wt;
            sum.z += c.z * wt;
            wsum += wt;
        }
    }
    dst[i0] = wsum > 1e-9f ? make_float4(sum.x / wsum, sum.y / wsum, sum.z / wsum, 0.f) : c0;
}

__global__ void k_remodulate(const float4* __restrict__ illum, const float* __restrict__ film, uint32_t npix,
                             float* __restrict__ rgb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const float* f = film + (size_t)RT_FILM_FLOATS * i;
    const float4 l = illum[i];
    rgb[3 * (size_t)i] = l.x * fmaxf(f[RT_FILM_ALBEDO], 5e-2f) + f[RT_FILM_SPECULAR];
    rgb[3 * (size_t)i + 1] = l.y * fmaxf(f[RT_FILM_ALBEDO + 1], 5e-2f) + f[RT_FILM_SPECULAR + 1];
    rgb[3 * (size_t)i + 2] = l.z * fmaxf(f[RT_FILM_ALBEDO + 2], 5e-2f) + f[RT_FILM_SPECULAR + 2];
}

int fail_film(int code, const std::string& msg) {
    accum_error() = msg;
    return code;
}

#define FM_TRY(expr)                                                                                  \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail_film(e_ == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA,              \
                             std::string(#expr) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

struct Bufs {
    cudaStream_t st;
    std::vector<void*> p;
    explicit Bufs(cudaStream_t s) : st(s) {}
    ~Bufs() {
        for (void* q : p) pool_free(q, st);
    }
    template <class T>
    cudaError_t get(T** out, size_t n) {
        void* v = nullptr;
        cudaError_t e = pool_alloc(&v, std::max<size_t>(n, 1) * sizeof(T), st);
        if (e == cudaSuccess) p.push_back(v);
        *out = (T*)v;
        return e;
    }
};

}  // namespace

// Film decode into a device array (18 floats per pixel) on `st`.
int film_decode_device(const double* accum, const float* aux, uint32_t npix, float* film, cudaStream_t st) {
    k_film_decode<<<(npix + FB - 1) / FB, FB, 0, st>>>(accum, aux, npix, film);
    FM_TRY(cudaGetLastError());
    return RT_OK;
}

// Denoise a device film into device rgb (3 floats per pixel) on `st`;
// synchronises `st` once (median depth on the host).
int denoise_device(const float* film, uint32_t w, uint32_t h, float* rgb, cudaStream_t st) {
    const uint32_t npix = w * h;
    if (npix == 0) return RT_OK;
    Bufs B(st);
    float4 *ill[2], *guide;
    float* id;
    FM_TRY(B.get(&ill[0], npix));
    FM_TRY(B.get(&ill[1], npix));
    FM_TRY(B.get(&guide, npix));
    FM_TRY(B.get(&id, npix));
    k_denoise_prep<<<(npix + FB - 1) / FB, FB, 0, st>>>(film, npix, ill[0], guide, id);
    FM_TRY(cudaGetLastError());
    // Depth scale: the median positive depth (denoise.rs:56-64).
    std::vector<float4> g(npix);
    FM_TRY(cudaMemcpyAsync(g.data(), guide, 16ull * npix, cudaMemcpyDeviceToHost, st));
    FM_TRY(cudaStreamSynchronize(st));
    std::vector<float> depths;
    depths.reserve(npix);
    for (const float4& v : g)
        if (v.w > 0.0f) depths.push_back(v.w);
    float scale = 1.0f;
    if (!depths.empty()) {
        std::nth_element(depths.begin(), depths.begin() + depths.size() / 2, depths.end());
        scale = depths[depths.size() / 2];
    }
    scale = std::max(scale, 1e-3f);
    float sigma = 8.0f;
    dim3 grid((w + 15) / 16, (h + 15) / 16);
    int cur = 0;
    for (int it = 0; it < 5; it++) {
        k_atrous<<<grid, 256, 0, st>>>(ill[cur], guide, id, w, h, 1 << it, 1.0f / (sigma * sigma), 1.0f / scale,
                                       ill[cur ^ 1]);
        cur ^= 1;
        sigma *= 0.5f;
    }
    k_remodulate<<<(npix + FB - 1) / FB, FB, 0, st>>>(ill[cur], film, npix, rgb);
    FM_TRY(cudaGetLastError());
    FM_TRY(cudaStreamSynchronize(st));
    return RT_OK;
}

}  // namespace rt

using namespace rt;

extern "C" int rt_denoise_film(const float* film, uint32_t width, uint32_t height, float* rgb) {
    if (!film || !rgb) return fail_film(RT_ERR_INVALID, "NULL argument");
    const uint64_t npix = (uint64_t)width * height;
    if (npix == 0) return RT_OK;
    if (npix >= (1ull << 31)) return fail_film(RT_ERR_INVALID, "image too large");
    cudaStream_t st;
    FM_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    int rc = RT_OK;
    {
        Bufs B(st);
        float *d_film = nullptr, *d_rgb = nullptr;
        cudaError_t e = B.get(&d_film, RT_FILM_FLOATS * npix);
        if (e == cudaSuccess) e = B.get(&d_rgb, 3 * npix);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_film, film, 4ull * RT_FILM_FLOATS * npix, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            rc = fail_film(e == cudaErrorMemoryAllocation ? RT_ERR_OOM : RT_ERR_CUDA, cudaGetErrorString(e));
        } else {
            rc = denoise_device(d_film, width, height, d_rgb, st);
            if (!rc && cudaMemcpyAsync(rgb, d_rgb, 12ull * npix, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                rc = fail_film(RT_ERR_CUDA, "denoise read-back failed");
        }
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

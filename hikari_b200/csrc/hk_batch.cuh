// Config-2 BSDF batch kernel, one instantiation per top-level BSDF type; the
// instantiations are spread over hk_batch_*.cu so they compile in parallel.
#pragma once
#include "hk_kernels.h"
#include "hk_shading.cuh"

namespace hk {

// Config-2 BSDF batch: per record Sample (wo, weight, pdf of the sampled
// direction, measure), Eval and Pdf at the given wo with ESolidAngle.
// One instantiation per top-level BSDF type (the host picks the id's type),
// so a launch carries only that BSDF's code.
template <int BT, bool kTex>
__global__ void bsdf_batch_kernel(DevScene S, int bsdf, uint64_t n, const float *wi, const float *u2, const float *u1,
                                  const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w,
                                  float *s_pdf, int32_t *s_m, float *e_rgb, float *p_pdf) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        BRec r;
        r.wi = v3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        r.wo = v3(0, 0, 0);
        r.measure = kMeasureUnknown;
        r.eta = 0.0f;
        r.tex = kTex;
        r.tu = kTex ? uv[2 * i] : 0.0f;
        r.tv = kTex ? uv[2 * i + 1] : 0.0f;
        r.duv = (kTex && duv) ? make_float4(duv[4 * i], duv[4 * i + 1], duv[4 * i + 2], duv[4 * i + 3])
                              : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        V3 w = bsdf_sample_t<BT>(S.bsdfs, bsdf, r, u2[2 * i], u2[2 * i + 1], u1 ? u1[i] : 0.0f);
        if (s_wo) { s_wo[3 * i] = r.wo.x; s_wo[3 * i + 1] = r.wo.y; s_wo[3 * i + 2] = r.wo.z; }
        if (s_w) { s_w[3 * i] = w.x; s_w[3 * i + 1] = w.y; s_w[3 * i + 2] = w.z; }
        if (s_m) s_m[i] = r.measure;
        if (s_pdf) s_pdf[i] = all_zero(w) ? 0.0f : bsdf_pdf_t<BT>(S.bsdfs, bsdf, r);
        BRec q;
        q.wi = r.wi;
        q.wo = v3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        q.measure = kMeasureSolidAngle;
        q.eta = 0.0f;
        q.tex = kTex;
        q.tu = r.tu;
        q.tv = r.tv;
        q.duv = r.duv;
        if (e_rgb) {
            V3 e = bsdf_eval_t<BT>(S.bsdfs, bsdf, q);
            e_rgb[3 * i] = e.x; e_rgb[3 * i + 1] = e.y; e_rgb[3 * i + 2] = e.z;
        }
        if (p_pdf) p_pdf[i] = bsdf_pdf_t<BT>(S.bsdfs, bsdf, q);
    }
}

template <int BT>
cudaError_t launch_bsdf_batch_t(const DevScene &S, int bsdf, uint64_t n, const float *wi, const float *u2, const float *u1,
                                const float *wo, const float *uv, const float *duv, float *s_wo, float *s_w, float *s_pdf,
                                int32_t *s_m, float *e_rgb, float *p_pdf, int grid, cudaStream_t st) {
    if (uv) bsdf_batch_kernel<BT, true><<<grid, 256, 0, st>>>(S, bsdf, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf);
    else bsdf_batch_kernel<BT, false><<<grid, 256, 0, st>>>(S, bsdf, n, wi, u2, u1, wo, uv, duv, s_wo, s_w, s_pdf, s_m, e_rgb, p_pdf);
    return cudaGetLastError();
}

}  // namespace hk

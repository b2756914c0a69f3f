/* Headless render driver over the reference's own classes, compiled into the
 * oracle's build of the reference (oracle/ref_build.py).  It does what
 * src/Main.cpp's Render (:46-147) does without the preview window (Screen,
 * OpenGL): load the scene XML through the reference parser, call the
 * integrator's Preprocess, hand out 32x32 image blocks from the reference
 * BlockGenerator, render each block on a host thread with that thread's clone
 * of the sampler (Sampler::Prepare seeds it from the block offset) through
 * the per-pixel loop of RenderBlock (:11-44), and merge each block into the
 * result with ImageBlock::Put.  The reference runs the block loop with
 * tbb::parallel_for; here std::thread workers pull block indices from an
 * atomic counter.  Used by tests (path-level pins of the oracle) and as the
 * timed CPU baseline; never by the library. */
#include <core\Common.hpp>
#include <core\Object.hpp>
#include <core\Parser.hpp>
#include <core\Scene.hpp>
#include <core\Camera.hpp>
#include <core\Integrator.hpp>
#include <core\Sampler.hpp>
#include <core\Block.hpp>
#include <core\Bitmap.hpp>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

using namespace Hikari;

namespace {
thread_local std::string g_err;

/* RenderBlock (src/Main.cpp:11-44): per pixel, per sample: pixel sample,
 * aperture sample, camera ray, Li, Put -- in this order, since the sampler's
 * stream is consumed in it. */
void render_block(const Scene *pScene, Sampler *pSampler, ImageBlock &Block) {
    const Camera *pCamera = pScene->GetCamera();
    const Integrator *pIntegrator = pScene->GetIntegrator();
    const Point2i Offset = Block.GetOffset();
    const Vector2i Size = Block.GetSize();
    Block.Clear();
    for (int y = 0; y < Size.y(); ++y)
        for (int x = 0; x < Size.x(); ++x)
            for (uint32_t i = 0; i < pSampler->GetSampleCount(); ++i) {
                Point2f PixelSample = Point2f(float(x + Offset.x()), float(y + Offset.y())) + pSampler->Next2D();
                Point2f ApertureSample = pSampler->Next2D();
                Ray3f R;
                Color3f Value = pCamera->SampleRay(R, PixelSample, ApertureSample);
                Value *= pIntegrator->Li(pScene, pSampler, R);
                Block.Put(PixelSample, Value);
            }
}
}  // namespace

extern "C" {

const char *hr_last_error(void) { return g_err.c_str(); }

/* LoadFromXML (src/core/Parser.cpp:9) with the scene file's directory on the
 * file resolver, as src/Main.cpp:166 does; NULL on error (hr_last_error). */
void *hr_scene_load(const char *xml_path) {
    try {
        filesystem::path P(xml_path);
        GetFileResolver()->prepend(P.parent_path());
        Object *o = LoadFromXML(xml_path);
        if (!o || o->GetClassType() != Object::EClassType::EScene) {
            delete o;
            g_err = "the XML root is not a scene";
            return nullptr;
        }
        return o;
    } catch (const std::exception &e) {
        g_err = e.what();
        return nullptr;
    }
}

void hr_scene_free(void *s) { delete (Object *)s; }

/* out: width, height, samples per pixel, film border */
void hr_scene_info(void *s, int *out4) {
    const Scene *S = (const Scene *)s;
    const Vector2i sz = S->GetCamera()->GetOutputSize();
    ImageBlock probe(Vector2i(1, 1), S->GetCamera()->GetReconstructionFilter());
    out4[0] = sz.x();
    out4[1] = sz.y();
    out4[2] = (int)S->GetSampler()->GetSampleCount();
    out4[3] = probe.GetBorderSize();
}

/* Render like src/Main.cpp:46-147.  blocks: NULL for the BlockGenerator's
 * own order (the first max_blocks blocks it hands out, all when
 * max_blocks <= 0), else nblocks block indices, row-major over the 32x32
 * block grid.  film_rgbw: (H+2B) x (W+2B) x 4 floats, the result ImageBlock
 * (RGB and filter weight).  Returns the render time in seconds (block loop
 * only, as the reference's timer), or < 0 on error. */
double hr_render(void *s, int nthreads, int max_blocks, const int *blocks, int nblocks, float *film_rgbw) {
    try {
        Scene *S = (Scene *)s;
        const Camera *pCamera = S->GetCamera();
        const Vector2i OutputSize = pCamera->GetOutputSize();
        S->GetIntegrator()->Preprocess(S);
        BlockGenerator Gen(OutputSize, HIKARI_BLOCK_SIZE);
        ImageBlock Result(OutputSize, pCamera->GetReconstructionFilter());
        Result.Clear();
        const int bx = (OutputSize.x() + HIKARI_BLOCK_SIZE - 1) / HIKARI_BLOCK_SIZE;
        const int total = Gen.GetBlockCount();
        const int count = blocks ? nblocks : (max_blocks > 0 ? std::min(max_blocks, total) : total);
        std::atomic<int> next(0);
        std::mutex gen_lock;
        if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
        auto t0 = std::chrono::steady_clock::now();
        auto worker = [&] {
            ImageBlock Block(Vector2i(HIKARI_BLOCK_SIZE), pCamera->GetReconstructionFilter());
            std::unique_ptr<Sampler> pSampler(S->GetSampler()->Clone());
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= count) break;
                if (blocks) {
                    const int b = blocks[i];
                    const int x0 = (b % bx) * HIKARI_BLOCK_SIZE, y0 = (b / bx) * HIKARI_BLOCK_SIZE;
                    Block.SetOffset(Point2i(x0, y0));
                    Block.SetSize(Point2i(std::min(HIKARI_BLOCK_SIZE, OutputSize.x() - x0),
                                          std::min(HIKARI_BLOCK_SIZE, OutputSize.y() - y0)));
                } else {
                    std::lock_guard<std::mutex> g(gen_lock);
                    Gen.Next(Block);
                }
                pSampler->Prepare(Block);
                render_block(S, pSampler.get(), Block);
                Result.Put(Block);
            }
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
        for (auto &t : th) t.join();
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (film_rgbw) {
            const int H = (int)Result.rows(), W = (int)Result.cols();
            for (int y = 0; y < H; ++y)
                for (int x = 0; x < W; ++x)
                    for (int c = 0; c < 4; ++c) film_rgbw[(4 * ((size_t)y * W + x)) + c] = Result.coeff(y, x)[c];
        }
        return secs;
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1.0;
    }
}

}  // extern "C"

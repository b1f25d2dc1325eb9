// TEST DRIVER for the drop-in: renders one PBRT scene through the reference's
// own frontend with the reference CpuBackend and with yr::CudaBackend as
// implemented by integration/yaoray_cuda_backend.cpp (linked in place of the
// reference's CUDA stub), and writes both films for comparison.
//
//   yaoray_dropin scene.pbrt out_prefix
// writes out_prefix.cpu.film / out_prefix.cuda.film (raw FilmPixel arrays)
// and prints one JSON line with stats and the progress-callback pass count.
#include <yaoray/backends/cpu/cpu_backend.hpp>
#include <yaoray/frontend/pbrt/pbrt_scene.hpp>
#include <yaoray/frontend/pbrt/scene_compiler.hpp>
#include <yaoray/runtime/backend.hpp>
#include <yaoray/runtime/cuda_stub_backend.hpp>

#include <cstdio>
#include <fstream>
#include <iostream>

namespace {

bool WriteFilm(const yr::Film& film, const std::string& path) {
    std::ofstream out(path, std::ios::binary);
    out.write(reinterpret_cast<const char*>(film.Pixels().data()),
              static_cast<std::streamsize>(film.Pixels().size() * sizeof(yr::FilmPixel)));
    return static_cast<bool>(out);
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: yaoray_dropin scene.pbrt out_prefix\n";
        return 2;
    }
    auto loaded = yr::LoadPbrtScene(argv[1]);
    if (!loaded.scene) {
        std::cerr << "load failed\n";
        return 1;
    }
    auto compiled = yr::CompilePbrtScene(*loaded.scene);
    if (!compiled.scene) {
        std::cerr << "compile failed\n";
        return 1;
    }
    const std::string prefix = argv[2];
    double seconds[2] = {0, 0};
    std::uint64_t rays[2] = {0, 0};
    int passes = 0;
    for (int which = 0; which < 2; ++which) {
        yr::RenderJob job{*compiled.scene, compiled.settings};
        job.settings.requested_backend = which == 0 ? yr::RenderBackendKind::Cpu : yr::RenderBackendKind::Cuda;
        std::unique_ptr<yr::RenderBackend> backend;
        if (which == 0) backend = std::make_unique<yr::CpuBackend>();
        else backend = std::make_unique<yr::CudaBackend>();
        yr::BackendPrepareResult prepared = backend->Prepare(std::move(job));
        if (!prepared.ok) {
            std::cerr << (which ? "cuda" : "cpu") << " prepare failed: " << prepared.error << "\n";
            return 1;
        }
        yr::RenderRequest request;
        if (which == 1) {
            request.progress_callback = [&](const yr::RenderProgress& p, const yr::Film& f) {
                ++passes;
                (void)p;
                (void)f;
                return yr::RenderProgressDecision{};
            };
        }
        yr::RenderResult result = backend->Render(*prepared.scene, request);
        if (!result.ok || !result.film) {
            std::cerr << (which ? "cuda" : "cpu") << " render failed: " << result.error << "\n";
            return 1;
        }
        seconds[which] = result.stats.elapsed_seconds;
        rays[which] = result.stats.rays_traced;
        if (!WriteFilm(*result.film, prefix + (which ? ".cuda.film" : ".cpu.film"))) return 1;
    }
    std::printf("{\"cpu_seconds\": %.6f, \"cuda_seconds\": %.6f, \"cpu_rays\": %llu, \"cuda_rays\": %llu, "
                "\"cuda_progress_calls\": %d}\n",
                seconds[0], seconds[1], static_cast<unsigned long long>(rays[0]),
                static_cast<unsigned long long>(rays[1]), passes);
    return 0;
}

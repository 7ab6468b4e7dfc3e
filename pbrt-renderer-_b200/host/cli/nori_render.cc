// nori_render — render a Nori XML scene on the GPU and write the linear HDR
// mean image: OpenEXR when the output name ends in .exr, PFM otherwise.
//   nori_render scene.xml [spp] [out.exr|out.pfm]
#include <cstdio>
#include <cstdlib>
#include <string>

#include "nori/nori.h"

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s scene.xml [spp] [out.exr|out.pfm]\n", argv[0]);
        return 2;
    }
    try {
        std::unique_ptr<nori::NoriObject> root(nori::loadFromXML(argv[1]));
        auto *scene = static_cast<nori::Scene *>(root.get());
        auto *gi = dynamic_cast<nori::GPUIntegrator *>(scene->getIntegrator());
        if (!gi) throw nori::NoriException("the scene has no path_mis / direct integrator");
        uint32_t spp = argc > 2 ? (uint32_t)std::atoi(argv[2]) : (uint32_t)scene->getSampler()->getSampleCount();
        std::string out = argc > 3 ? argv[3] : "render.pfm";
        gi->preprocess(scene);
        nori::RenderResult r = gi->render(spp);
        std::vector<float> img = r.mean();
        if (out.size() > 4 && out.compare(out.size() - 4, 4, ".exr") == 0) {
            nori::writeEXR(out, r.width, r.height, img.data());
        } else {
            FILE *f = std::fopen(out.c_str(), "wb");
            if (!f) throw nori::NoriException("cannot write " + out);
            std::fprintf(f, "PF\n%d %d\n-1.0\n", r.width, r.height);
            for (int y = r.height - 1; y >= 0; y--)
                std::fwrite(&img[(size_t)y * r.width * 3], 4, (size_t)r.width * 3, f);
            std::fclose(f);
        }
        std::printf("%s: %dx%d, %u spp, %.2f ms on the GPU (%.1f Mpaths/s)\n", out.c_str(), r.width, r.height, spp,
                    r.stats.ms_total, r.stats.paths / (r.stats.ms_total * 1e3));
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "Error: %s\n", e.what());
        return 1;
    }
}

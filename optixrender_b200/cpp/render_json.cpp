// render_json - headless replacement of the reference's viewer (main.cpp:165-265):
// loads a scene JSON (models/test.json schema), renders `frames` progressive
// launches, and writes the RGBA8 image (DownloadPixels) as PNG and binary PPM
// and the float colour buffer as a PFM.
//
//   render_json scene.json out_prefix [frames] [spp]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "optixrender.hpp"

static bool write_ppm(const char* path, const std::vector<uint32_t>& px, int w, int h) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    std::fprintf(f, "P6\n%d %d\n255\n", w, h);
    for (int y = h - 1; y >= 0; y--)  // row 0 of the frame buffer is the bottom
        for (int x = 0; x < w; x++) {
            uint32_t p = px[size_t(y) * w + x];
            unsigned char rgb[3] = {uint8_t(p & 255), uint8_t((p >> 8) & 255), uint8_t((p >> 16) & 255)};
            std::fwrite(rgb, 1, 3, f);
        }
    std::fclose(f);
    return true;
}

static bool write_pfm(const char* path, const std::vector<float>& rgba, int w, int h) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    std::fprintf(f, "PF\n%d %d\n-1.0\n", w, h);  // bottom-to-top rows, little endian
    for (size_t i = 0; i < size_t(w) * h; i++) std::fwrite(&rgba[i * 4], 4, 3, f);
    std::fclose(f);
    return true;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s scene.json out_prefix [frames] [spp]\n", argv[0]);
        return 2;
    }
    int frames = argc > 3 ? std::atoi(argv[3]) : 1;
    try {
        rt::Scene scene;
        rt::Options opts;
        rt::Camera cam;
        scene.LoadFromJson(argv[1], opts, cam);
        if (argc > 4) opts.spp = std::atoi(argv[4]);
        opts.progressive = 1;
        rt::Renderer renderer(scene, opts);
        renderer.SetCamera(cam);
        for (int i = 0; i < frames; i++) renderer.Render();
        std::vector<uint32_t> px(size_t(opts.width) * opts.height);
        std::vector<float> lin(px.size() * 4);
        renderer.DownloadPixels(px.data());
        renderer.DownloadLinear(lin.data());
        std::string pre = argv[2];
        if (!write_ppm((pre + ".ppm").c_str(), px, opts.width, opts.height) ||
            !write_pfm((pre + ".pfm").c_str(), lin, opts.width, opts.height) ||
            rt_write_png((pre + ".png").c_str(), px.data(), opts.width, opts.height) != RT_OK) {
            std::fprintf(stderr, "could not write %s.*\n", argv[2]);
            return 1;
        }
        rt_render_stats st = renderer.Stats();
        std::printf("rendered %dx%d, %d frame(s) x %d spp in %.2f ms (last frame)\n", opts.width, opts.height, frames,
                    opts.spp, st.ms_total);
    } catch (const rt::Error& e) {
        std::fprintf(stderr, "error %d: %s\n", e.code, e.what());
        return 1;
    }
    return 0;
}

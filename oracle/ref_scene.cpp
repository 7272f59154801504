// ref_scene.cpp - extern "C" access to HdrTexture::CalculateHdrCache of the
// reference renderer (core/src/Scene.cpp:217-313), compiled from the reference
// source.  TEST INFRASTRUCTURE ONLY (see ref_driver.cpp).
#include "Scene.h"

extern "C" void ref_env_cache(const float* rgba, int32_t w, int32_t h, float* cache) {
    HdrTexture t("");  // an empty name loads nothing; the image is set below
    t.hdr = new float[size_t(w) * h * 4];
    for (size_t i = 0; i < size_t(w) * h * 4; i++) t.hdr[i] = rgba[i];
    t.width = w;
    t.height = h;
    t.comp = 4;
    t.CalculateHdrCache();
    for (size_t i = 0; i < size_t(w) * h; i++) {
        cache[i * 4 + 0] = t.cache[i * 4 + 0];
        cache[i * 4 + 1] = t.cache[i * 4 + 1];
        cache[i * 4 + 2] = t.cache[i * 4 + 2];
        cache[i * 4 + 3] = 0.0f;
    }
}

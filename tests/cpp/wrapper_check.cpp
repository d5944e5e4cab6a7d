// Drives PathTracerB200 (tests/cpp/PathTracerB200.h) the way the reference's
// viewport drives class PathTracer: a HostMesh of the reference's own types,
// a CameraGpu, RenderParamsGpu defaults with a fixed sample budget, render,
// readback.  Reads the scene from a binary file the Python test writes and
// writes the image back, so the test can compare it with the Python API's
// render of the same scene.
//
//   wrapper_check <scene.bin> <image.bin>
//
// scene.bin: int32 w, h, spp, triangle count n, material count m, texture
// count t; then n HostTriangle-equivalents as 24 floats (v0 v1 v2 n0 n1 n2 uv0
// uv1 uv2) + one uint32 material index each; m MaterialGpu records; t
// TextureDescGpu records; one CameraGpu.
#include "PathTracerB200.h"

#include <cstdio>
#include <vector>

int main(int argc, char** argv)
{
    if (argc != 3) {
        std::fprintf(stderr, "usage: wrapper_check <scene.bin> <image.bin>\n");
        return 2;
    }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (f == nullptr) {
        return 2;
    }
    int32_t hdr[6] = {};
    if (std::fread(hdr, sizeof(int32_t), 6, f) != 6 || hdr[0] <= 0 || hdr[1] <= 0 || hdr[3] < 0 || hdr[4] < 0 ||
        hdr[5] < 0) {
        return 2;
    }
    HostMesh mesh;
    mesh.triangles.resize(static_cast<size_t>(hdr[3]));
    for (HostTriangle& t : mesh.triangles) {
        float v[24];
        uint32_t mi = 0;
        if (std::fread(v, sizeof(float), 24, f) != 24 || std::fread(&mi, sizeof(mi), 1, f) != 1) {
            return 2;
        }
        t.v0 = Vec3{v[0], v[1], v[2]};
        t.v1 = Vec3{v[3], v[4], v[5]};
        t.v2 = Vec3{v[6], v[7], v[8]};
        t.n0 = Vec3{v[9], v[10], v[11]};
        t.n1 = Vec3{v[12], v[13], v[14]};
        t.n2 = Vec3{v[15], v[16], v[17]};
        t.uv0 = Vec2{v[18], v[19]};
        t.uv1 = Vec2{v[20], v[21]};
        t.uv2 = Vec2{v[22], v[23]};
        t.materialIndex = mi;
    }
    mesh.materials.resize(static_cast<size_t>(hdr[4]));
    if (hdr[4] > 0 && std::fread(mesh.materials.data(), sizeof(MaterialGpu), mesh.materials.size(), f) !=
            mesh.materials.size()) {
        return 2;
    }
    mesh.textures.resize(static_cast<size_t>(hdr[5]));
    if (hdr[5] > 0 && std::fread(mesh.textures.data(), sizeof(TextureDescGpu), mesh.textures.size(), f) !=
            mesh.textures.size()) {
        return 2;
    }
    CameraGpu cam{};
    if (std::fread(&cam, sizeof(CameraGpu), 1, f) != 1) {
        return 2;
    }
    std::fclose(f);

    PathTracerB200 pt(0);
    RenderParamsGpu params{}; // the reference's defaults
    params.backgroundR = params.backgroundG = params.backgroundB = 0.1f;
    params.maxPathDepth = 6;
    params.minSamples = hdr[2];
    params.maxSamplesPerPixel = hdr[2];
    if (!pt.configure(hdr[0], hdr[1], mesh) || !pt.setCamera(cam) || !pt.setRenderParams(params)) {
        std::fprintf(stderr, "setup failed: %s\n", pt.lastError());
        return 1;
    }
    const CameraGpu back = pt.lastSampleCamera();
    if (std::memcmp(&back, &cam, sizeof(CameraGpu)) != 0) {
        std::fprintf(stderr, "lastSampleCamera differs from setCamera\n");
        return 1;
    }
    pt.resetAccumulation();
    if (!pt.render(0)) {
        std::fprintf(stderr, "render failed: %s\n", pt.lastError());
        return 1;
    }
    std::vector<float> rgba;
    std::vector<uint32_t> counts;
    if (!pt.readback(rgba, counts)) {
        return 1;
    }
    std::FILE* o = std::fopen(argv[2], "wb");
    if (o == nullptr || std::fwrite(rgba.data(), sizeof(float), rgba.size(), o) != rgba.size() ||
        std::fwrite(counts.data(), sizeof(uint32_t), counts.size(), o) != counts.size()) {
        return 1;
    }
    std::fclose(o);
    return 0;
}

// PathTracer-shaped C++ wrapper over the C ABI (include/pt_b200.h): what a
// maintainer of the reference would add to PathTracerLib so that call sites of
// class PathTracer (PathTracerLib/src/PathTracer.h:30-152) keep their shape with
// the GL/Qt parts removed.  It takes the reference's own records -- HostMesh
// (Application/src/MeshBuilder/HostMesh.h:9-28), CameraGpu (CameraGpu.h:5-16),
// RenderParamsGpu (RenderTypes.h:15-28) -- and passes them through unchanged;
// the static_asserts pin the byte layouts the ABI relies on.  Compiled against
// the reference headers and run by tests/test_gpu_cxx_wrapper.py.
#pragma once

#include "CameraGpu.h"
#include "MeshBuilder/HostMesh.h"
#include "RenderTypes.h"
#include "pt_b200.h"

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

static_assert(sizeof(MaterialGpu) == sizeof(pt_material), "MaterialGpu and pt_material differ");
static_assert(sizeof(TextureDescGpu) == sizeof(pt_texture), "TextureDescGpu and pt_texture differ");
static_assert(sizeof(CameraGpu) == sizeof(pt_camera), "CameraGpu and pt_camera differ");
static_assert(sizeof(RenderParamsGpu) == 44 && sizeof(pt_render_params) > sizeof(RenderParamsGpu),
    "pt_render_params starts with RenderParamsGpu");
static_assert(offsetof(pt_render_params, relative_error_threshold) == offsetof(RenderParamsGpu, relativeErrorThreshold),
    "RenderParamsGpu prefix of pt_render_params");

class PathTracerB200 {
public:
    explicit PathTracerB200(int device = 0)
    {
        if (pt_create(&r_, device) != PT_OK) {
            throw std::runtime_error(pt_last_error(nullptr));
        }
    }
    ~PathTracerB200() { pt_destroy(r_); }
    PathTracerB200(const PathTracerB200&) = delete;
    PathTracerB200& operator=(const PathTracerB200&) = delete;

    // PathTracer::configure (PathTracer.h:45-51) without the GL PBOs.
    bool configure(int width, int height, const HostMesh& mesh)
    {
        if (pt_configure(r_, width, height) != PT_OK) {
            return false;
        }
        w_ = width;
        h_ = height;
        return rebuildMeshScene(mesh);
    }
    // PathTracer::rebuildMeshScene (PathTracer.h:130-132): HostTriangle -> SoA.
    bool rebuildMeshScene(const HostMesh& mesh)
    {
        const size_t n = mesh.triangles.size();
        pos_.resize(9 * n);
        nrm_.resize(9 * n);
        uv_.resize(6 * n);
        mat_.resize(n);
        for (size_t i = 0; i < n; ++i) {
            const HostTriangle& t = mesh.triangles[i];
            const Vec3 v[3] = {t.v0, t.v1, t.v2};
            const Vec3 nn[3] = {t.n0, t.n1, t.n2};
            const Vec2 q[3] = {t.uv0, t.uv1, t.uv2};
            for (int k = 0; k < 3; ++k) {
                pos_[9 * i + 3 * k] = v[k].x;
                pos_[9 * i + 3 * k + 1] = v[k].y;
                pos_[9 * i + 3 * k + 2] = v[k].z;
                nrm_[9 * i + 3 * k] = nn[k].x;
                nrm_[9 * i + 3 * k + 1] = nn[k].y;
                nrm_[9 * i + 3 * k + 2] = nn[k].z;
                uv_[6 * i + 2 * k] = q[k].x;
                uv_[6 * i + 2 * k + 1] = q[k].y;
            }
            mat_[i] = t.materialIndex;
        }
        pt_mesh m{static_cast<uint32_t>(n), pos_.data(), nrm_.data(), uv_.data(), mat_.data(),
            static_cast<uint32_t>(mesh.materials.size()), reinterpret_cast<const pt_material*>(mesh.materials.data()),
            static_cast<uint32_t>(mesh.textures.size()), reinterpret_cast<const pt_texture*>(mesh.textures.data())};
        return pt_set_mesh(r_, &m) == PT_OK;
    }
    // PathTracer::setCamera / lastSampleCamera (PathTracer.h:101-103).
    bool setCamera(const CameraGpu& c) { return pt_set_camera(r_, reinterpret_cast<const pt_camera*>(&c)) == PT_OK; }
    CameraGpu lastSampleCamera() const
    {
        CameraGpu c{};
        pt_get_camera(r_, reinterpret_cast<pt_camera*>(&c));
        return c;
    }
    // The setters of PathTracer.h:73-124 as one record; the extension tail
    // stays zero, which selects the reference's behaviour.
    bool setRenderParams(const RenderParamsGpu& p)
    {
        pt_render_params q{};
        std::memcpy(&q, &p, sizeof(RenderParamsGpu));
        return pt_set_params(r_, &q) == PT_OK;
    }
    void resetAccumulation() { pt_reset(r_); }
    // The worker thread's render loop, synchronously: `waves` adaptive waves (0 = until done).
    bool render(int waves) { return pt_render(r_, waves) == PT_OK; }
    // Headless replacement of the PBO publish: running-mean RGBA per pixel.
    bool readback(std::vector<float>& rgba, std::vector<uint32_t>& counts)
    {
        rgba.resize(4 * static_cast<size_t>(w_) * h_);
        counts.resize(static_cast<size_t>(w_) * h_);
        return pt_readback(r_, rgba.data(), counts.data(), nullptr) == PT_OK;
    }
    const char* lastError() const { return pt_last_error(r_); }

private:
    pt_renderer* r_ = nullptr;
    int w_ = 0;
    int h_ = 0;
    std::vector<float> pos_, nrm_, uv_;
    std::vector<uint32_t> mat_;
};

// The REFERENCE's scene generator for the parity checker: L-system text ->
// symbol string -> turtle -> Hermite spline frames -> lofted tubes.  Built into
// oracle/_ref/libptref_gen.so by oracle/Makefile (target refgen).  Test and
// benchmark infrastructure only: the product never loads it.
//
// Compiled unchanged from the reference tree:
//   - LSystemLib (LSystemEvaluator::evaluate, LSystemEvaluator.h:24-27, and the
//     parser under LSystemLib/src);
//   - Application/src/Procedural/Turtle.cpp (turtleExecute, :275-282);
//   - Application/src/Procedural/Spline.cpp (SplinePath::buildFromSegment,
//     computeLoftFrames, :102-255).
// Restated here because their files include the manifold library, which the
// checkout does not carry:
//   - buildLoftHostMeshFromFrames and its helpers (Loft.cpp:23-155);
//   - rotateYawPitchRoll / applyRootTransform for host meshes
//     (ProceduralMeshBuilder.cpp:211-253);
//   - the loft branch of ProceduralMeshBuilder::buildHostMesh
//     (ProceduralMeshBuilder.cpp:266-330): every turtle segment whose spline
//     has an arc length above 1e-6 is lofted; the manifold validity filter
//     (always satisfied by these tubes) and the sphere fallback for
//     zero-length segments (counted in `skipped`) are left out.
#include "Geometry/MathCore.h"
#include "LSystemEvaluator.h"
#include "MeshBuilder/HostMesh.h"
#include "Procedural/Spline.h"
#include "Procedural/Turtle.h"

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

namespace {

struct LoftCorner {
    Vec3 position{};
    Vec3 normal{};
    Vec2 uv{};
};

// Loft.cpp:23-32.
Vec3 ringVertex(const PathFrame& frame, int segmentIndex, int circularSegments)
{
    const float angle = static_cast<float>(segmentIndex) * 6.283185307f / static_cast<float>(circularSegments);
    const float c = std::cos(angle);
    const float s = std::sin(angle);
    return vecAdd3(frame.position,
        vecAdd3(vecScale3(frame.normal, c * frame.radius), vecScale3(frame.binormal, s * frame.radius)));
}

// Loft.cpp:34-40.
Vec2 planarCapUv(int segmentIndex, int circularSegments)
{
    const float angle = static_cast<float>(segmentIndex) * 6.283185307f / static_cast<float>(circularSegments);
    return Vec2{0.5f + 0.5f * std::sin(angle), 0.5f + 0.5f * std::cos(angle)};
}

// Loft.cpp:66-94.
LoftCorner sideWallCorner(const PathFrame& frame, int segment, int circularSegments, float vCoord)
{
    const int geomSegment = segment < circularSegments ? segment : 0;
    const Vec3 position = ringVertex(frame, geomSegment, circularSegments);
    const Vec3 normal = vecNormalize3(vecSub3(position, frame.position));
    const float uCoord = static_cast<float>(segment) / static_cast<float>(circularSegments);
    return LoftCorner{position, normal, Vec2{uCoord, vCoord}};
}

LoftCorner capRimCorner(const PathFrame& frame, int segment, int circularSegments, float normalSign)
{
    return LoftCorner{ringVertex(frame, segment, circularSegments), vecNormalize3(vecScale3(frame.tangent, normalSign)),
        planarCapUv(segment, circularSegments)};
}

LoftCorner capCenterCorner(const PathFrame& frame, float normalSign)
{
    return LoftCorner{frame.position, vecNormalize3(vecScale3(frame.tangent, normalSign)), Vec2{0.5f, 0.5f}};
}

void appendTriangle(HostMesh& mesh, const LoftCorner& c0, const LoftCorner& c1, const LoftCorner& c2)
{
    HostTriangle t{};
    t.v0 = c0.position;
    t.v1 = c1.position;
    t.v2 = c2.position;
    t.n0 = c0.normal;
    t.n1 = c1.normal;
    t.n2 = c2.normal;
    t.uv0 = c0.uv;
    t.uv1 = c1.uv;
    t.uv2 = c2.uv;
    mesh.triangles.push_back(t);
}

// Loft.cpp:108-155: side walls ring by ring, then the two caps interleaved.
void loftFromFrames(const std::vector<PathFrame>& frames, int circularSegments, HostMesh& mesh)
{
    if (frames.size() < 2 || circularSegments < 3) {
        return;
    }
    const int ringCount = static_cast<int>(frames.size());
    const float invRingSpan = 1.0f / static_cast<float>(ringCount - 1);
    for (int ring = 0; ring < ringCount - 1; ++ring) {
        const float v0 = static_cast<float>(ring) * invRingSpan;
        const float v1 = static_cast<float>(ring + 1) * invRingSpan;
        const PathFrame& f0 = frames[static_cast<size_t>(ring)];
        const PathFrame& f1 = frames[static_cast<size_t>(ring + 1)];
        for (int segment = 0; segment < circularSegments; ++segment) {
            const LoftCorner a00 = sideWallCorner(f0, segment, circularSegments, v0);
            const LoftCorner a01 = sideWallCorner(f0, segment + 1, circularSegments, v0);
            const LoftCorner a10 = sideWallCorner(f1, segment, circularSegments, v1);
            const LoftCorner a11 = sideWallCorner(f1, segment + 1, circularSegments, v1);
            appendTriangle(mesh, a00, a01, a10);
            appendTriangle(mesh, a01, a11, a10);
        }
    }
    const PathFrame& start = frames.front();
    const PathFrame& end = frames.back();
    const LoftCorner startCenter = capCenterCorner(start, -1.0f);
    const LoftCorner endCenter = capCenterCorner(end, 1.0f);
    for (int segment = 0; segment < circularSegments; ++segment) {
        const int next = (segment + 1) % circularSegments;
        appendTriangle(mesh, startCenter, capRimCorner(start, next, circularSegments, -1.0f),
            capRimCorner(start, segment, circularSegments, -1.0f));
        appendTriangle(mesh, endCenter, capRimCorner(end, segment, circularSegments, 1.0f),
            capRimCorner(end, next, circularSegments, 1.0f));
    }
}

// ProceduralMeshBuilder.cpp:211-241.
constexpr float kDegToRad = 0.0174532925f;

Vec3 rotateAroundAxis(Vec3 value, Vec3 axis, float radians)
{
    const Vec3 unitAxis = vecNormalize3(axis);
    const float c = std::cos(radians);
    const float s = std::sin(radians);
    const float dot = vecDot3(unitAxis, value);
    const Vec3 cross = vecMake3(unitAxis.y * value.z - unitAxis.z * value.y, unitAxis.z * value.x - unitAxis.x * value.z,
        unitAxis.x * value.y - unitAxis.y * value.x);
    return vecAdd3(vecAdd3(vecScale3(value, c), vecScale3(cross, s)), vecScale3(unitAxis, dot * (1.0f - c)));
}

Vec3 rotateYawPitchRoll(Vec3 v, const float* rotationDeg)
{
    if (std::fabs(rotationDeg[0]) > 1.0e-6f) {
        v = rotateAroundAxis(v, Vec3{0.0f, 1.0f, 0.0f}, rotationDeg[0] * kDegToRad);
    }
    if (std::fabs(rotationDeg[1]) > 1.0e-6f) {
        v = rotateAroundAxis(v, Vec3{1.0f, 0.0f, 0.0f}, rotationDeg[1] * kDegToRad);
    }
    if (std::fabs(rotationDeg[2]) > 1.0e-6f) {
        v = rotateAroundAxis(v, Vec3{0.0f, 0.0f, 1.0f}, rotationDeg[2] * kDegToRad);
    }
    return v;
}

struct GenResult {
    HostMesh mesh;
    std::vector<uint32_t> triSegment;   // turtle segment of each triangle
    std::vector<uint32_t> segMaterial;  // numeric material id of each lofted segment
    std::vector<PathFrame> frames;      // loft frames of every lofted segment, in order
    std::vector<uint32_t> frameStart;   // per lofted segment: first frame
    std::vector<uint32_t> symbolCount;
    double ms[4] = {0.0, 0.0, 0.0, 0.0}; // L-system, turtle, spline frames, loft + root transform
    int skipped = 0;
    std::string error;
};

double msSince(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

} // namespace

extern "C" {

// Runs the reference generator.  rotationDeg: yaw, pitch, roll (degrees) of the
// root transform; translation: 3 floats.  Returns a handle (never NULL; check
// refgen_error for a parse failure).
void* refgen_build(const char* definition, int iterations, unsigned long long seed, const float* rotationDeg,
    const float* translation, int circularSegments, int samplesPerSpan, float hermiteTension, float defaultStep,
    float defaultRadius)
{
    GenResult* g = new GenResult();
    try {
        auto t0 = std::chrono::steady_clock::now();
        const LSystemEvaluationResult eval =
            LSystemEvaluator::evaluate(std::string(definition), static_cast<std::size_t>(iterations), seed);
        g->ms[0] = msSince(t0);
        g->symbolCount.push_back(static_cast<uint32_t>(eval.generation.size()));
        t0 = std::chrono::steady_clock::now();
        TurtleParams tp{};
        tp.defaultStepLength = defaultStep;
        tp.defaultRadius = defaultRadius;
        const TurtleOutput out = turtleExecute(eval.generation, tp);
        g->ms[1] = msSince(t0);
        std::vector<std::vector<PathFrame>> segFrames;
        t0 = std::chrono::steady_clock::now();
        for (const TurtleSegment& seg : out.segments) {
            SplinePath path;
            if (!path.buildFromSegment(seg, hermiteTension) || path.totalArcLength() <= 1e-6f) {
                segFrames.emplace_back();
                ++g->skipped;
                continue;
            }
            segFrames.push_back(path.computeLoftFrames(samplesPerSpan));
        }
        g->ms[2] = msSince(t0);
        t0 = std::chrono::steady_clock::now();
        for (size_t k = 0; k < out.segments.size(); ++k) {
            const std::vector<PathFrame>& frames = segFrames[k];
            if (frames.size() < 2) {
                continue;
            }
            const size_t before = g->mesh.triangles.size();
            loftFromFrames(frames, circularSegments, g->mesh);
            for (size_t i = before; i < g->mesh.triangles.size(); ++i) {
                HostTriangle& t = g->mesh.triangles[i];
                const Vec3 tr = Vec3{translation[0], translation[1], translation[2]};
                t.v0 = vecAdd3(rotateYawPitchRoll(t.v0, rotationDeg), tr);
                t.v1 = vecAdd3(rotateYawPitchRoll(t.v1, rotationDeg), tr);
                t.v2 = vecAdd3(rotateYawPitchRoll(t.v2, rotationDeg), tr);
                t.n0 = rotateYawPitchRoll(t.n0, rotationDeg);
                t.n1 = rotateYawPitchRoll(t.n1, rotationDeg);
                t.n2 = rotateYawPitchRoll(t.n2, rotationDeg);
                g->triSegment.push_back(static_cast<uint32_t>(k));
            }
            uint32_t mat = 0;
            try {
                mat = static_cast<uint32_t>(std::stoul(out.segments[k].materialId));
            } catch (const std::exception&) {
                mat = 0;
            }
            g->segMaterial.push_back(mat);
            g->frameStart.push_back(static_cast<uint32_t>(g->frames.size()));
            g->frames.insert(g->frames.end(), frames.begin(), frames.end());
        }
        g->frameStart.push_back(static_cast<uint32_t>(g->frames.size()));
        g->ms[3] = msSince(t0);
    } catch (const std::exception& e) {
        g->error = e.what();
    }
    return g;
}

void refgen_destroy(void* h)
{
    delete static_cast<GenResult*>(h);
}

const char* refgen_error(void* h)
{
    return static_cast<GenResult*>(h)->error.c_str();
}

// counts[0] triangles, [1] lofted segments, [2] frames, [3] skipped segments, [4] symbols
void refgen_counts(void* h, int* counts)
{
    const GenResult* g = static_cast<GenResult*>(h);
    counts[0] = static_cast<int>(g->mesh.triangles.size());
    counts[1] = static_cast<int>(g->segMaterial.size());
    counts[2] = static_cast<int>(g->frames.size());
    counts[3] = g->skipped;
    counts[4] = g->symbolCount.empty() ? 0 : static_cast<int>(g->symbolCount[0]);
}

// Stage times in ms: L-system, turtle, spline frames, loft + root transform.
void refgen_times(void* h, double* ms)
{
    std::memcpy(ms, static_cast<GenResult*>(h)->ms, sizeof(double) * 4);
}

// Triangles: positions 9, normals 9, uvs 6 floats; turtle segment per triangle.
void refgen_triangles(void* h, float* positions, float* normals, float* uvs, uint32_t* segment)
{
    const GenResult* g = static_cast<GenResult*>(h);
    for (size_t i = 0; i < g->mesh.triangles.size(); ++i) {
        const HostTriangle& t = g->mesh.triangles[i];
        const Vec3 v[3] = {t.v0, t.v1, t.v2}, n[3] = {t.n0, t.n1, t.n2};
        const Vec2 q[3] = {t.uv0, t.uv1, t.uv2};
        for (int k = 0; k < 3; ++k) {
            positions[9 * i + 3 * k] = v[k].x;
            positions[9 * i + 3 * k + 1] = v[k].y;
            positions[9 * i + 3 * k + 2] = v[k].z;
            normals[9 * i + 3 * k] = n[k].x;
            normals[9 * i + 3 * k + 1] = n[k].y;
            normals[9 * i + 3 * k + 2] = n[k].z;
            uvs[6 * i + 2 * k] = q[k].x;
            uvs[6 * i + 2 * k + 1] = q[k].y;
        }
        segment[i] = g->triSegment[i];
    }
}

// Loft frames before the root transform: 13 floats each (position, tangent,
// normal, binormal, radius); frameStart: lofted segments + 1 offsets;
// materials: numeric material id per lofted segment.
void refgen_frames(void* h, float* frames, uint32_t* frameStart, uint32_t* materials)
{
    const GenResult* g = static_cast<GenResult*>(h);
    for (size_t i = 0; i < g->frames.size(); ++i) {
        const PathFrame& f = g->frames[i];
        const float v[13] = {f.position.x, f.position.y, f.position.z, f.tangent.x, f.tangent.y, f.tangent.z,
            f.normal.x, f.normal.y, f.normal.z, f.binormal.x, f.binormal.y, f.binormal.z, f.radius};
        std::memcpy(frames + 13 * i, v, sizeof(v));
    }
    std::memcpy(frameStart, g->frameStart.data(), g->frameStart.size() * sizeof(uint32_t));
    if (!g->segMaterial.empty()) {
        std::memcpy(materials, g->segMaterial.data(), g->segMaterial.size() * sizeof(uint32_t));
    }
}

} // extern "C"

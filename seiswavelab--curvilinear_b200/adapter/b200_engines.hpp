// Reference-side binding: the two engine adapters a SeisWave Lab maintainer adds beside the
// reference's own CUDA engines to run its sessions on libswl_b200 (a third compute backend).
//
// Include this after the reference's mesh and receiver types
// (src/two_d/PointKernels2D.hpp, include/Seis2D/CurvilinearSolver2D.hpp,
// src/three_d/PointKernels3D.hpp, include/Seis3D/CurvilinearSolver.hpp) and link -lswl_b200.
// The adapters take exactly what the reference hands its CudaEngine
// (src/two_d/CudaEngine2D.hpp:7-8) and CudaEngine3D (src/three_d/CudaEngine3D.hpp:9): a non-owning
// Point::MeshT / Point::Mesh view of the model arrays, the receivers and a device index.  The mesh
// mirror is filled field by field (toMesh2D / toMesh3D); the engine copies every array at create.
// Errors come back as std::runtime_error with the library's message, as the reference's checked()
// does (src/common/CudaSupport.cuh:5-8).
#pragma once
#include "swl_b200.h"
#include <cstdint>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace swl_b200 {

// Point::MeshT<Real> (src/two_d/PointKernels2D.hpp:14-27) -> swl_mesh2d.  Real is double or float:
// the reference converts its stored arrays to the session precision before building the mesh.
template <class MeshT> swl_mesh2d toMesh2D(const MeshT &m) {
    using Real = std::remove_cv_t<std::remove_pointer_t<decltype(m.a)>>;
    static_assert(std::is_same_v<Real, double> || std::is_same_v<Real, float>, "MeshT<double> or MeshT<float>");
    swl_mesh2d g{};
    g.nx = m.nx, g.nz = m.nz, g.count = int64_t(m.count), g.h = double(m.h);
    g.a = m.a, g.b = m.b, g.jac = m.jac, g.normals = m.normals;
    g.lambda = m.lambda, g.mu = m.mu, g.rho = m.rho, g.source = m.source, g.damping = m.damping;
    for (int a = 0; a < 3; ++a) g.source_direction[a] = double(m.sourceDirection[a]);
    g.source_gradient[0] = m.sourceGradient[0], g.source_gradient[1] = m.sourceGradient[1];
    g.mechanisms = m.mechanisms, g.field_count = m.fieldCount;
    g.cpml_x = m.cpmlX, g.cpml_z = m.cpmlZ, g.cpml_width_x = m.cpmlWidthX, g.cpml_width_z = m.cpmlWidthZ;
    g.cpml_count = int64_t(m.cpmlCount);
    for (int l = 0; l < 3; ++l) g.rates[l] = double(m.rates[l]), g.delta_p[l] = m.deltaP[l], g.delta_s[l] = m.deltaS[l];
    g.precision = g.array_precision = std::is_same_v<Real, float> ? SWL_FP32 : SWL_FP64;
    return g;
}

// Point::Mesh (src/three_d/PointKernels3D.hpp:13-21) -> swl_mesh3d, computed in `precision`.
template <class Mesh> swl_mesh3d toMesh3D(const Mesh &m, int32_t precision = SWL_FP64) {
    swl_mesh3d g{};
    g.nx = m.nx, g.ny = m.ny, g.nz = m.nz, g.count = int64_t(m.count);
    g.h = m.h, g.lambda = m.lambda, g.mu = m.mu, g.density = m.density;
    g.metrics = m.metrics, g.normals = m.normals, g.jacobian = m.jacobian, g.source = m.source, g.damping = m.damping;
    g.material_lambda = m.materialLambda, g.material_mu = m.materialMu, g.material_density = m.materialDensity;
    for (int a = 0; a < 3; ++a) g.source_direction[a] = m.sourceDirection[a], g.source_gradient[a] = m.sourceGradient[a];
    g.source_amplitude = m.sourceAmplitude;
    g.precision = precision;
    return g;
}

// Padded node of each receiver, as CudaEngine computes it (Point::index(mesh, x + 3, z + 3),
// src/two_d/CudaEngine2D.cu:139).
template <class MeshT, class Receiver> std::vector<int64_t> receiverNodes2D(const MeshT &m, const std::vector<Receiver> &receivers) {
    std::vector<int64_t> nodes;
    nodes.reserve(receivers.size());
    for (const auto &r : receivers) nodes.push_back(int64_t(r.x + 3) + int64_t(m.nx) * (r.z + 3));
    return nodes;
}

inline void checked(swl_status s) {
    if (s != SWL_OK) throw std::runtime_error(swl_last_error());
}

// The 2D engine: the same constructor arguments as CudaEngine.  Receivers are the reference's
// Receiver (x, z logical node indices; CudaEngine2D.cu:139 adds the ghost width).
class B200Engine2D {
  public:
    template <class MeshT, class Receiver>
    B200Engine2D(const MeshT &m, const std::vector<Receiver> &receivers, int device) {
        const swl_mesh2d g = toMesh2D(m);
        const std::vector<int64_t> nodes = receiverNodes2D(m, receivers);
        checked(swl2d_create(&g, nodes.data(), int32_t(nodes.size()), device, &e_));
    }
    ~B200Engine2D() { swl2d_destroy(e_); }
    B200Engine2D(const B200Engine2D &) = delete;
    B200Engine2D &operator=(const B200Engine2D &) = delete;
    swl2d_engine *get() const { return e_; }
    void step(double time, double dt, double frequency, double scale, int step) { checked(swl2d_step(e_, time, dt, frequency, scale, step)); }
    void rollback() { checked(swl2d_rollback(e_)); }
    void reset() { checked(swl2d_reset(e_)); }
    std::size_t residentBytes() const { return std::size_t(swl2d_resident_bytes(e_)); }

  private:
    swl2d_engine *e_{};
};

// The 3D engine: the same constructor arguments as CudaEngine3D.  ReceiverTrace3D carries the
// padded grid index of its node (include/Seis3D/CurvilinearSolver.hpp:129-134).
class B200Engine3D {
  public:
    template <class Mesh, class Trace>
    B200Engine3D(const Mesh &m, const std::vector<Trace> &receivers, int device, int32_t precision = SWL_FP64) {
        const swl_mesh3d g = toMesh3D(m, precision);
        std::vector<int64_t> nodes;
        nodes.reserve(receivers.size());
        for (const auto &r : receivers) nodes.push_back(int64_t(r.gridIndex));
        checked(swl3d_create(&g, nodes.data(), int32_t(nodes.size()), device, &e_));
    }
    ~B200Engine3D() { swl3d_destroy(e_); }
    B200Engine3D(const B200Engine3D &) = delete;
    B200Engine3D &operator=(const B200Engine3D &) = delete;
    swl3d_engine *get() const { return e_; }
    void step(double time, double dt, double frequency, int step) { checked(swl3d_step(e_, time, dt, frequency, step)); }
    void rollback() { checked(swl3d_rollback(e_)); }
    void resetFields() { checked(swl3d_reset(e_)); }

  private:
    swl3d_engine *e_{};
};

} // namespace swl_b200

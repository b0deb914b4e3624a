// Compiled by tests/test_adapter.py against the reference's own mesh and receiver types (its
// headers, read-only) and the reference-side adapters of seiswavelab--curvilinear_b200/adapter:
// every field of Point::MeshT<double>, Point::MeshT<float> and the 3D Point::Mesh must land in
// the matching field of the C mirror, receiver nodes must equal the reference's Point::index, and
// an engine request without a usable GPU must come back as an exception, not a crash.
#include "PointKernels2D.hpp"
#include "Seis2D/CurvilinearSolver2D.hpp"
#include "PointKernels3D.hpp"
#include "Seis3D/CurvilinearSolver.hpp"
#include "b200_engines.hpp"
#include <cstdio>
#include <cstring>
#include <vector>

static int failures = 0;
#define CHECK(c)                                                                                                       \
    do {                                                                                                               \
        if (!(c)) std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c), ++failures;                                 \
    } while (0)

template <class Real> void check2d() {
    namespace P = Seis2D::Curvilinear::Point;
    constexpr int nx = 20, nz = 16;
    std::vector<std::vector<Real>> arrays(24, std::vector<Real>(2 * nx * nz));
    int next = 0;
    auto arr = [&]() { return arrays[next++].data(); };
    P::MeshT<Real> m;
    m.nx = nx, m.nz = nz, m.count = std::size_t(nx) * nz, m.h = Real(2.5);
    m.a = arr(), m.b = arr(), m.jac = arr(), m.normals = arr(), m.lambda = arr(), m.mu = arr(), m.rho = arr();
    m.source = arr(), m.damping = arr();
    m.sourceDirection[0] = Real(0.25), m.sourceDirection[1] = Real(0.5), m.sourceDirection[2] = Real(0.75);
    m.sourceGradient[0] = arr(), m.sourceGradient[1] = arr();
    m.mechanisms = 3, m.fieldCount = 18;
    m.cpmlX = arr(), m.cpmlZ = arr(), m.cpmlWidthX = 4, m.cpmlWidthZ = 3, m.cpmlCount = 1234;
    for (int l = 0; l < 3; ++l) m.rates[l] = Real(10 + l), m.deltaP[l] = arr(), m.deltaS[l] = arr();
    const swl_mesh2d g = swl_b200::toMesh2D(m);
    CHECK(g.nx == nx && g.nz == nz && g.count == int64_t(m.count) && g.h == double(m.h));
    CHECK(g.a == m.a && g.b == m.b && g.jac == m.jac && g.normals == m.normals);
    CHECK(g.lambda == m.lambda && g.mu == m.mu && g.rho == m.rho && g.source == m.source && g.damping == m.damping);
    for (int a = 0; a < 3; ++a) CHECK(g.source_direction[a] == double(m.sourceDirection[a]));
    CHECK(g.source_gradient[0] == m.sourceGradient[0] && g.source_gradient[1] == m.sourceGradient[1]);
    CHECK(g.mechanisms == m.mechanisms && g.field_count == m.fieldCount);
    CHECK(g.cpml_x == m.cpmlX && g.cpml_z == m.cpmlZ && g.cpml_width_x == m.cpmlWidthX && g.cpml_width_z == m.cpmlWidthZ);
    CHECK(g.cpml_count == int64_t(m.cpmlCount));
    for (int l = 0; l < 3; ++l) CHECK(g.rates[l] == double(m.rates[l]) && g.delta_p[l] == m.deltaP[l] && g.delta_s[l] == m.deltaS[l]);
    const int32_t want = std::is_same_v<Real, float> ? SWL_FP32 : SWL_FP64;
    CHECK(g.precision == want && g.array_precision == want);
    std::vector<Seis2D::Curvilinear::Receiver> rec(3);
    rec[0].x = 0, rec[0].z = 0, rec[1].x = 7, rec[1].z = 2, rec[2].x = nx - 7, rec[2].z = nz - 7;
    const auto nodes = swl_b200::receiverNodes2D(m, rec);
    for (std::size_t r = 0; r < rec.size(); ++r) CHECK(nodes[r] == int64_t(P::index(m, rec[r].x + 3, rec[r].z + 3)));
    bool threw = false;
    try {
        swl_b200::B200Engine2D e(m, rec, 0);
    } catch (const std::runtime_error &ex) {
        threw = std::strlen(ex.what()) > 0;
    }
    CHECK(threw); // no usable GPU here: an error status, turned into an exception
}

void check3d() {
    namespace P = Seis3D::Curvilinear::Point;
    std::vector<std::vector<double>> arrays(12, std::vector<double>(64));
    int next = 0;
    auto arr = [&]() { return arrays[next++].data(); };
    P::Mesh m;
    m.nx = 20, m.ny = 18, m.nz = 16, m.count = std::size_t(20) * 18 * 16;
    m.h = 10, m.lambda = 1.5e9, m.mu = 1e9, m.density = 2000;
    m.metrics = arr(), m.normals = arr(), m.jacobian = arr(), m.source = arr(), m.damping = arr();
    m.materialLambda = arr(), m.materialMu = arr(), m.materialDensity = arr();
    m.sourceDirection[0] = 0.1, m.sourceDirection[1] = 0.2, m.sourceDirection[2] = 0.97, m.sourceAmplitude = 3e9;
    for (int a = 0; a < 3; ++a) m.sourceGradient[a] = arr();
    const swl_mesh3d g = swl_b200::toMesh3D(m, SWL_FP32);
    CHECK(g.nx == m.nx && g.ny == m.ny && g.nz == m.nz && g.count == int64_t(m.count));
    CHECK(g.h == m.h && g.lambda == m.lambda && g.mu == m.mu && g.density == m.density);
    CHECK(g.metrics == m.metrics && g.normals == m.normals && g.jacobian == m.jacobian && g.source == m.source && g.damping == m.damping);
    CHECK(g.material_lambda == m.materialLambda && g.material_mu == m.materialMu && g.material_density == m.materialDensity);
    for (int a = 0; a < 3; ++a) CHECK(g.source_direction[a] == m.sourceDirection[a] && g.source_gradient[a] == m.sourceGradient[a]);
    CHECK(g.source_amplitude == m.sourceAmplitude && g.precision == SWL_FP32);
    std::vector<Seis3D::Curvilinear::ReceiverTrace3D> rec(2);
    rec[0].gridIndex = P::index(m, 3, 3, 3), rec[1].gridIndex = P::index(m, 9, 8, 3);
    bool threw = false;
    try {
        swl_b200::B200Engine3D e(m, rec, 0);
    } catch (const std::runtime_error &ex) {
        threw = std::strlen(ex.what()) > 0;
    }
    CHECK(threw);
}

int main() {
    check2d<double>();
    check2d<float>();
    check3d();
    std::printf(failures ? "FAILED %d\n" : "OK\n", failures);
    return failures ? 1 : 0;
}

// Host-side model construction (FP64) for the 2D and 3D sessions: the parameter structures,
// the GSLS fit, the PCHIP terrain profile and the model arrays that the engines consume.
// Everything here restates the reference's session initialisation; each function names the
// lines it follows.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace swl::host {

// --------------------------------------------------------------------- GSLS (Gsls.hpp/.cpp)
struct GslsSettings {
    bool enabled{};
    int mechanisms{3};
    double minFrequency{5}, maxFrequency{100}, referenceFrequency{30}, qp{100}, qs{60};
};
struct GslsMaterial {
    int mechanisms{};
    double pRelaxed{}, sRelaxed{}, pUnrelaxed{}, sUnrelaxed{}, maxRelativeQError{};
    std::array<double, 3> rates{}, deltaP{}, deltaS{};
};
void validateGsls(const GslsSettings &);
GslsMaterial fitGsls(double vp, double vs, double rho, double qp, double qs, const GslsSettings &);
double gslsQuality(const GslsMaterial &, bool shear, double frequency);

// ---------------------------------------------------------------- terrain (SurfaceProfile.cpp)
class SurfaceProfile {
  public:
    explicit SurfaceProfile(const std::vector<std::array<double, 2>> &points);
    std::array<double, 2> sample(double x) const; // elevation, slope
  private:
    std::vector<std::array<double, 2>> points_;
    std::vector<double> slopes_;
};

// ------------------------------------------------------------------------- 2D parameters
struct Layer2D {
    double thickness{}, vp{}, vs{}, density{}, qp{100}, qs{60};
};
// Seis2D::Curvilinear::Parameters (include/Seis2D/CurvilinearSolver2D.hpp:29-57)
struct Params2D {
    int precision{0};
    int nx{200}, nz{200};
    double spacing{2.5}, vp{3000}, vs{1700}, density{2200};
    double relief{10}, wavelength{400}, flattenDepth{}, frequency{30}, duration{1}, cfl{.8}, forcePerLength{2e5};
    int sourceX{-1}, sourceZ{40}, maxSteps{5000};
    int sourceKind{0}; // 0 directional force, 1 isotropic moment
    std::array<double, 3> sourceDirection{0, 0, 1};
    double momentPerLength{2e6}, sourceSigmaM{}, sourceRadiusM{};
    bool absorbing{true};
    int spongeX{16}, spongeZ{16};
    double spongeStrength{3};
    int absorber{0}; // 0 sponge, 1 CFS-PML
    double cpmlReflection{1e-4}, cpmlKappaMax{3}, cpmlFrequency{};
    bool externalAbsorption{};
    int receiverStart{2}, receiverCount{96}, receiverStride{2}, receiverDepth{1};
    double sampleIntervalMs{};
    bool layered{};
    GslsSettings attenuation;
    bool importedSurface{};
    double surfaceDatum{};
    std::vector<std::array<double, 2>> surfaceSamples;
    // FP64 node geometry (coordinates, metrics, Jacobian, normals) built on this CUDA device
    // (-1: the largest) instead of on the host; not part of the reference's Parameters.
    bool deviceGeometry{false};
    int geometryDevice{-1};
    // the engine's stage-kernel segment by occupancy rule instead of timing runs (a server's shots)
    bool segmentRule{false};
    std::vector<Layer2D> layers{{20, 1500, 700, 2050, 100, 60}, {50, 2500, 1300, 2250, 100, 60}, {0, 4000, 2300, 2650, 100, 60}};
};

// All FP64 model arrays of a 2D session (padded (nx+6)x(nz+6), x fastest).
struct Model2D {
    int nx{}, nz{};          // padded
    int modelOffsetX{};      // storage columns before the logical model
    int logicalNx{}, logicalNz{};
    double h{}, flattenDepth{}, maxMetric{}, minJacobian{}, maxEdge{};
    std::vector<double> coordinates, normals; // 2 per node
    std::vector<double> metricA, metricB, jacobian, vp, vs, density, lambda, mu, source, damping, qp, qs;
    std::vector<double> sourceGradient[2];
    std::vector<double> cpmlX, cpmlZ;
    int cpmlWidthX{}, cpmlWidthZ{};
    std::int64_t cpmlCount{};
    int mechanisms{}, fieldCount{5};
    std::array<double, 3> rates{};
    std::vector<double> deltaP[3], deltaS[3];
    std::array<double, 3> sourceDirection{};
    double scale{};           // force (or moment) per length / h^2
    double dt{};
    int total{};
    int sourceX{}, sourceZ{}; // storage-logical source node (after the absorber offset)
    std::vector<std::int64_t> receiverNodes; // padded node index per receiver
    std::vector<std::array<double, 2>> receiverPositions;
    // diagnostics of the plan
    double ppw{}, waveDt{}, dampingDt{}, sourceDt{}, relaxationDt{}, cpmlDt{}, maxRelativeQError{};
    double sourceWeightSum{}, sourceRmsRadiusM{};
    double recordDt{};
    std::size_t recordSamples{};
};

// Simulation::initialize (src/two_d/CurvilinearSolver2D.cpp:151-540), model part.  Throws
// std::runtime_error with the reference's messages on invalid parameters.
Model2D buildModel2D(const Params2D &);

// ------------------------------------------------------------------------- 3D parameters
struct Layer3D {
    double thickness{}, vp{}, vs{}, density{};
    double qp{-1}, qs{-1}; // GSLS quality factors of the layer (< 0: the session's attenuation.qp/qs)
};
struct SurfaceGrid3D {
    int nx{}, ny{};
    double spacing{}, originX{}, originY{}, datum{};
    std::vector<double> elevations;
    bool empty() const { return elevations.empty(); }
    double elevation(double x, double y) const;
    double displacement(double x, double y) const { return datum - elevation(x, y); }
};
// Seis3D::Curvilinear::SimulationParameters (include/Seis3D/CurvilinearSolver.hpp:70-95)
struct Params3D {
    int precision{0};
    int nx{28}, ny{24}, nz{28};
    double spacing{10}, vp{3000}, vs{1700}, density{2200};
    bool layered{};
    int layerDepthMode{0}; // 0 grid index, 1 below surface, 2 datum
    std::vector<Layer3D> layers;
    double frequency{12};
    int sourceX{-1}, sourceY{-1}, sourceZ{3};
    int sourceKind{0};
    std::array<double, 3> sourceDirection{0, 0, 1};
    double sourceForce{2e8}, sourceMoment{2e9};
    double duration{1};
    int maxSteps{5000};
    double cfl{.8};
    double relief{20}, wavelength{300}, flattenDepth{};
    SurfaceGrid3D surfaceGrid;
    // receivers: kind 0 auto x-line, 1 x-line, 2 y-line, 3 grid
    int receiverKind{0}, receiverStartX{2}, receiverStartY{-1}, receiverZ{1}, receiverCountX{24}, receiverCountY{1},
        receiverStrideX{1}, receiverStrideY{1};
    bool absorbing{true};
    std::array<int, 3> absorbingCells{8, 6, 8};
    double absorbingStrength{3};
    // 0: the reference's quadratic sponge; 1: CFS-PML ADE slabs of the same widths (no counterpart
    // in the reference's 3D path; the 2D profiles of src/two_d/CfsPml2D.hpp:31-41 per axis)
    int absorber{0};
    double cpmlReflection{1e-4}, cpmlKappaMax{3}, cpmlFrequency{};
    // GSLS viscoelasticity (no counterpart in the reference's 3D path; the 2D fit and relaxation of
    // src/common/Gsls.cpp and src/two_d/PointKernels2D.hpp:161-168 with all six stress components)
    GslsSettings attenuation;
    int receiverLimit{1024}; // the reference caps traces at 1024; the engine has no such limit
    // FP64 node geometry built on this CUDA device (-1: the largest) instead of on the host
    bool deviceGeometry{false};
    int geometryDevice{-1};
    std::vector<std::string> layerNames; // MaterialLayer3D::name per layer (may be shorter: unnamed)
};
struct Model3D {
    int nx{}, ny{}, nz{};
    double h{}, lambda{}, mu{}, density{}, flattenDepth{};
    std::vector<double> coordinates; // 3 per node
    std::vector<double> metrics;     // 9 per node
    std::vector<double> jacobian, normals, source, damping, materialLambda, materialMu, materialDensity;
    std::vector<double> sourceGradient[3];
    std::array<double, 3> sourceDirection{};
    double sourceAmplitude{};
    double dt{};
    int total{};
    double minJacobian{}, maxMetricNorm{}, minCellLength{}, maxCellEdge{}, waveDt{}, dampingDt{}, sourceDt{}, ppw{};
    // CFS-PML: (d, kappa, alpha) per computational index along x, y, z; slab widths; memories
    std::vector<double> cpmlX, cpmlY, cpmlZ;
    std::array<int, 3> cpmlWidth{};
    std::int64_t cpmlCount{};
    std::vector<double> cpmlShape; // wx, wy, wz, memory count (as model array "cpmlShape")
    double cpmlDt{};
    // GSLS: mechanisms (0: elastic), relaxation rates, per-node strengths, dt bound
    int mechanisms{};
    std::array<double, 3> rates{};
    std::vector<double> deltaP[3], deltaS[3];
    std::vector<double> gslsRates; // the `mechanisms` rates (as model array "gslsRates")
    double relaxationDt{}, maxRelativeQError{};
    std::vector<std::int64_t> receiverNodes;
    std::vector<std::array<double, 3>> receiverPositions;
};
// CpuSimulation3D::initialize (src/three_d/CurvilinearSolver.cpp:301-442), model part.
Model3D buildModel3D(const Params3D &);
// src/two_d/CfsPml2D.hpp:31-41: (d, kappa, alpha) for `nodes` computational indices, a layer of
// `width` cells at both ends (`both`) or at the far end only; and the largest d/kappa + alpha.
std::vector<double> cpmlProfile(int nodes, int width, double h, double vp, double reflection, double kappa, double frequency,
                                bool both);
double cpmlRate(const std::vector<double> &profile);

} // namespace swl::host

// Test infrastructure only: drives the reference SeisWave Lab 3D nine-field solver
// (CpuSimulation3D), compiled from its own sources (oracle/Makefile), on a key/value case
// file and dumps the FP64 model arrays, receiver traces and final wavefields as
// little-endian float64 files.  The product never links or runs this program.
//
// Usage: ref3d <case.txt> <outdir> [steps] [threads] [dump_mesh 0|1] [warmup steps]
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <locale>
#include <map>
#include <memory>
#include <optional>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>
#ifdef SEIS3D_HAS_OPENMP
#include <omp.h>
#endif
#include <unistd.h>
#include "SeisCommon/SegyIo.hpp"
#define private public
#include "CurvilinearSolver.cpp"
#include "Seis3D/ReceiverIo.hpp"
#include "Seis3D/VtsWriter.hpp"
#undef private
#include "Seis3D/ModelIo3D.hpp"

using namespace Seis3D::Curvilinear;

namespace {
struct Case {
    std::map<std::string, std::vector<double>> kv;
    bool has(const char *k) const { return kv.count(k) != 0; }
    double num(const char *k, double fallback) const {
        auto it = kv.find(k);
        return it == kv.end() || it->second.empty() ? fallback : it->second[0];
    }
    const std::vector<double> &list(const char *k) const {
        static const std::vector<double> empty;
        auto it = kv.find(k);
        return it == kv.end() ? empty : it->second;
    }
};
Case readCase(const char *path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error(std::string("cannot open case file ") + path);
    in.imbue(std::locale::classic());
    Case c;
    std::string line;
    while (std::getline(in, line)) {
        if (auto p = line.find('#'); p != std::string::npos) line.resize(p);
        std::istringstream row(line);
        row.imbue(std::locale::classic());
        std::string key;
        if (!(row >> key)) continue;
        std::vector<double> values;
        double v;
        while (row >> v) values.push_back(v);
        c.kv[key] = std::move(values);
    }
    return c;
}
SimulationParameters parameters(const Case &c) {
    SimulationParameters p;
    p.nx = int(c.num("nx", p.nx));
    p.ny = int(c.num("ny", p.ny));
    p.nz = int(c.num("nz", p.nz));
    p.spacing = c.num("spacing", p.spacing);
    p.vp = c.num("vp", p.vp);
    p.vs = c.num("vs", p.vs);
    p.density = c.num("density", p.density);
    p.layeredMaterial = c.num("layered", 0) != 0;
    p.layerDepthMode = static_cast<LayerDepthMode3D>(int(c.num("layerDepthMode", 0)));
    if (c.has("layers")) {
        const auto &l = c.list("layers"); // thickness vp vs density per layer
        p.layers.clear();
        for (std::size_t i = 0; i + 4 <= l.size(); i += 4)
            p.layers.push_back({"layer" + std::to_string(i / 4), l[i], l[i + 1], l[i + 2], l[i + 3]});
    }
    p.dominantFrequency = c.num("frequency", p.dominantFrequency);
    p.sourceX = int(c.num("sourceX", p.sourceX));
    p.sourceY = int(c.num("sourceY", p.sourceY));
    p.sourceZ = int(c.num("sourceZ", p.sourceZ));
    p.source.kind = c.num("sourceKind", 0) ? SeisWave::SourceKind::IsotropicMoment
                                           : SeisWave::SourceKind::DirectionalForce;
    if (c.has("sourceDirection"))
        for (int a = 0; a < 3; ++a) p.source.direction[a] = c.list("sourceDirection").at(a);
    p.sourceForce = c.num("sourceForce", p.sourceForce);
    p.sourceMoment = c.num("sourceMoment", p.sourceMoment);
    p.duration = c.num("duration", p.duration);
    p.maxSteps = int(c.num("maxSteps", p.maxSteps));
    p.cflSafety = c.num("cfl", p.cflSafety);
    p.topographyAmplitude = c.num("relief", p.topographyAmplitude);
    p.topographyWavelength = c.num("wavelength", p.topographyWavelength);
    p.terrainTransitionDepth = c.num("flattenDepth", p.terrainTransitionDepth);
    if (c.has("demShape")) { // nx ny spacing originX originY datum
        const auto &d = c.list("demShape");
        p.surfaceGrid.nx = int(d.at(0));
        p.surfaceGrid.ny = int(d.at(1));
        p.surfaceGrid.spacing = d.at(2);
        p.surfaceGrid.originX = d.at(3);
        p.surfaceGrid.originY = d.at(4);
        p.surfaceGrid.datum = d.at(5);
        p.surfaceGrid.elevations = c.list("demElevations");
    }
    if (c.has("receiverArray")) { // kind startX startY z countX countY strideX strideY
        const auto &r = c.list("receiverArray");
        p.receiverArray.kind = static_cast<ReceiverArrayKind3D>(int(r.at(0)));
        p.receiverArray.startX = int(r.at(1));
        p.receiverArray.startY = int(r.at(2));
        p.receiverArray.z = int(r.at(3));
        p.receiverArray.countX = int(r.at(4));
        p.receiverArray.countY = int(r.at(5));
        p.receiverArray.strideX = int(r.at(6));
        p.receiverArray.strideY = int(r.at(7));
    }
    p.absorbingBoundary.enabled = c.num("absorbing", 1) != 0;
    if (c.has("absorbingCells"))
        for (int a = 0; a < 3; ++a) p.absorbingBoundary.cells[a] = int(c.list("absorbingCells").at(a));
    p.absorbingBoundary.strength = c.num("absorbingStrength", p.absorbingBoundary.strength);
    return p;
}
void write(const std::filesystem::path &dir, const std::string &name, const double *v, std::size_t n) {
    std::ofstream out(dir / name, std::ios::binary);
    out.write(reinterpret_cast<const char *>(v), static_cast<std::streamsize>(n * sizeof(double)));
    if (!out) throw std::runtime_error("write failed: " + name);
}
void write(const std::filesystem::path &dir, const std::string &name, const std::vector<double> &v) {
    write(dir, name, v.data(), v.size());
}
} // namespace

int main(int argc, char **argv) {
    try {
        if (argc < 3) {
            std::cerr << "usage: ref3d case.txt outdir [steps] [threads] [dump_mesh] [warmup]\n";
            return 2;
        }
        const auto c = readCase(argv[1]);
        const std::filesystem::path out(argv[2]);
        std::filesystem::create_directories(out);
        const int threads = argc > 4 ? std::atoi(argv[4]) : 1;
        const bool dumpMesh = argc > 5 ? std::atoi(argv[5]) != 0 : true;
        const auto p = parameters(c);
        CpuSimulation3D sim(BackendKind3D::Cpu);
        std::string error;
        const auto t0 = std::chrono::steady_clock::now();
        if (!sim.initialize(p, error, ComputeSettings3D{threads, -1})) {
            std::ofstream(out / "error.txt") << error << '\n';
            std::cerr << "initialize failed: " << error << '\n';
            return 3;
        }
        const double initMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        auto &s = *sim.impl_;
        const int steps = argc > 3 && std::atoi(argv[3]) >= 0 ? std::min(std::atoi(argv[3]), sim.totalSteps()) : sim.totalSteps();
        const auto &g = s.grid;
        const std::size_t count = g.coordinates.size();
        if (dumpMesh) {
            write(out, "coordinates.bin", reinterpret_cast<const double *>(g.coordinates.data()), 3 * count);
            write(out, "metrics.bin", reinterpret_cast<const double *>(g.inverseMetrics.data()), 9 * count);
            write(out, "jacobian.bin", g.jacobian);
            write(out, "normals.bin", reinterpret_cast<const double *>(g.surfaceNormal.data()), 3 * count);
            write(out, "source.bin", s.sourceWeights);
            write(out, "damping.bin", s.dampingRates);
            if (!s.sourceGradient[0].empty())
                for (int a = 0; a < 3; ++a) write(out, "sourceGradient" + std::to_string(a) + ".bin", s.sourceGradient[a]);
            if (!s.materialLambda.empty()) {
                write(out, "materialLambda.bin", s.materialLambda);
                write(out, "materialMu.bin", s.materialMu);
                write(out, "materialDensity.bin", s.materialDensity);
            }
        }
        const int warmup = argc > 6 ? std::max(0, std::atoi(argv[6])) : 0;
        if (warmup > 0 && !sim.advance(warmup, error)) std::cerr << "warm-up failed: " << error << '\n';
        const auto t1 = std::chrono::steady_clock::now();
        if (steps > 0 && !sim.advance(steps, error)) {
            std::ofstream(out / "error.txt") << error << '\n';
            std::cerr << "advance failed: " << error << '\n';
        }
        const double runMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
        for (int f = 0; f < 9; ++f) write(out, "field" + std::to_string(f) + ".bin", s.state.field[f]);
        std::vector<double> vx, vy, vz;
        for (const auto &r : sim.receivers()) {
            vx.insert(vx.end(), r.samplesVx.begin(), r.samplesVx.end());
            vy.insert(vy.end(), r.samplesVy.begin(), r.samplesVy.end());
            vz.insert(vz.end(), r.samples.begin(), r.samples.end());
        }
        write(out, "tracesVx.bin", vx);
        write(out, "tracesVy.bin", vy);
        write(out, "tracesVz.bin", vz);
        const bool files = argc > 8 && std::string(argv[8]) == "files";
        if (files) { // the reference's receiver CSV files (src/three_d/ReceiverIo.cpp): all components, and Vx+Vz
            std::string csvError;
            if (!writeReceiversCsv(sim, out / "receivers.csv", {true, true, true}, csvError) ||
                !writeReceiversCsv(sim, out / "receivers_xz.csv", {true, false, true}, csvError))
                std::ofstream(out / "csv_error.txt") << csvError << '\n';
        }
        if (files) { // writeModelVts3D (src/three_d/ModelIo3D.cpp:87-170) with this run's compute settings
            std::string modelError;
            if (!writeModelVts3D(sim, out / "model.vts", ComputeSettings3D{threads, -1}, modelError))
                std::ofstream(out / "model_error.txt") << modelError << '\n';
        }
        if (files) { // writeVts (src/three_d/VtsWriter.cpp) of the snapshot, default options and a reduced set
            std::string vtsError;
            VtsExportOptions3D some;
            some.fields = {false, false, true, false, true, false, false, false, true, false, false};
            some.includeMaterial = false;
            some.includeVelocityVector = false;
            const auto snap = sim.snapshot();
            if (!writeVts(snap, out / "snapshot.vts", VtsExportOptions3D{}, vtsError) ||
                !writeVts(snap, out / "snapshot_some.vts", some, vtsError))
                std::ofstream(out / "vts_error.txt") << vtsError << '\n';
        }
        if (files) { // the record view of src/three_d/ui/RecordView3D.cpp:5-6 through writeSegy
            SeisWave::RecordDataView data;
            data.dt = sim.dt();
            data.components = {"Vz", "Vx", "Vy"};
            for (const auto &trace : sim.receivers()) {
                SeisWave::TraceView t;
                t.position = trace.position;
                t.channels = {trace.samples, trace.samplesVx, trace.samplesVy};
                data.traces.push_back(t);
            }
            std::string segyError;
            if (!SeisWave::writeSegy(data, 0, out / "vz_ieee32.sgy", segyError, false) ||
                !SeisWave::writeSegy(data, 2, out / "vy_ieee64.sgy", segyError, true))
                std::ofstream(out / "segy_error.txt") << segyError << '\n';
        }
        const auto &d = sim.diagnostics();
        std::ofstream meta(out / "meta.txt");
        meta.imbue(std::locale::classic());
        meta << std::setprecision(17);
        meta << "nx " << g.nx << "\nny " << g.ny << "\nnz " << g.nz << "\ncount " << count << "\nh " << g.dx
             << "\ndt " << sim.dt() << "\ntotal " << sim.totalSteps() << "\nsteps " << sim.currentStep()
             << "\nlambda " << s.lambda << "\nmu " << s.mu << "\ndensity " << p.density << "\nlayered "
             << (s.materialLambda.empty() ? 0 : 1) << "\nreceivers " << sim.receivers().size() << "\nsamples "
             << (sim.receivers().empty() ? 0 : sim.receivers().front().samples.size()) << "\nreceiverIndex";
        for (const auto &r : sim.receivers()) meta << ' ' << r.gridIndex;
        meta << "\nflattenDepth " << g.terrainTransitionDepth << "\nminJacobian " << d.minJacobian
             << "\nmaxMetricNorm " << d.maxMetricNorm << "\nminCellLength " << d.minCellLength << "\nmaxCellEdge "
             << d.maxCellEdge << "\nwaveDt " << d.waveDtLimit << "\ndampingDt " << d.dampingDtLimit << "\nsourceDt "
             << d.sourceDtLimit << "\nenergy " << d.elasticEnergy << "\npeakEnergy " << d.peakEnergy
             << "\nmaxAbsVelocity " << d.maxAbsVelocity << "\ntractionRate " << d.maxTractionRateRelative
             << "\nfinite " << d.allFinite << "\nthreads " << s.backend.workerThreads << "\ninitMs " << initMs
             << "\nrunMs " << runMs << "\nmsPerStep " << (steps > 0 ? runMs / steps : 0.0) << "\nerror "
             << (error.empty() ? "none" : "set") << '\n';
        return 0;
    } catch (const std::exception &e) {
        std::cerr << "ref3d: " << e.what() << '\n';
        return 1;
    }
}

// Test infrastructure only: drives the reference SeisWave Lab 2D curvilinear solver,
// compiled from its own sources (oracle/Makefile), on a key/value case file and dumps
// the FP64 model arrays, raw receiver traces and final wavefields as little-endian
// float64 files.  Nothing in the product links or runs this program; tests use it as
// the parity truth and bench.py times it as the reference CPU arm.
//
// Usage: ref2d <case.txt> <outdir> [steps] [threads] [dump_mesh 0|1] [warmup steps] [cpu|cuda] [files]
//   files  : also write the reference's receiver CSV, SEG-Y, snapshot and model files (small cases only)
//   steps  : accepted RK4 steps to run (default: the session's total)
//   threads: ComputeSettings3D::cpuThreads (0 = reference default)
//
// The reference solver translation unit is included here so the driver can read the
// session's private model arrays (Simulation::Impl in CurvilinearSolver2D.cpp).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
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
#include <sstream>
#include <stdexcept>
#include <string>
#include <variant>
#include <vector>
#ifdef SEIS3D_HAS_OPENMP
#include <omp.h>
#endif
#include "SeisCommon/SegyIo.hpp"
#define private public
#include "CurvilinearSolver2D.cpp"
#undef private
#include "Seis2D/ModelIo2D.hpp"

using namespace Seis2D::Curvilinear;

namespace {
std::map<std::string, std::vector<double>> readCase(const char *path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error(std::string("cannot open case file ") + path);
    in.imbue(std::locale::classic());
    std::map<std::string, std::vector<double>> kv;
    std::string line;
    while (std::getline(in, line)) {
        if (auto c = line.find('#'); c != std::string::npos) line.resize(c);
        std::istringstream row(line);
        row.imbue(std::locale::classic());
        std::string key;
        if (!(row >> key)) continue;
        std::vector<double> values;
        double v;
        while (row >> v) values.push_back(v);
        kv[key] = std::move(values);
    }
    return kv;
}
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
Parameters parameters(const Case &c) {
    Parameters p;
    p.precision = c.num("precision", 0) ? Precision::Float32 : Precision::Float64;
    p.nx = int(c.num("nx", p.nx));
    p.nz = int(c.num("nz", p.nz));
    p.spacing = c.num("spacing", p.spacing);
    p.vp = c.num("vp", p.vp);
    p.vs = c.num("vs", p.vs);
    p.density = c.num("density", p.density);
    p.relief = c.num("relief", p.relief);
    p.wavelength = c.num("wavelength", p.wavelength);
    p.flattenDepth = c.num("flattenDepth", p.flattenDepth);
    p.frequency = c.num("frequency", p.frequency);
    p.duration = c.num("duration", p.duration);
    p.cfl = c.num("cfl", p.cfl);
    p.forcePerLength = c.num("forcePerLength", p.forcePerLength);
    p.sourceX = int(c.num("sourceX", p.sourceX));
    p.sourceZ = int(c.num("sourceZ", p.sourceZ));
    p.maxSteps = int(c.num("maxSteps", p.maxSteps));
    p.source.kind = c.num("sourceKind", 0) ? SeisWave::SourceKind::IsotropicMoment
                                           : SeisWave::SourceKind::DirectionalForce;
    if (c.has("sourceDirection"))
        for (int a = 0; a < 3; ++a) p.source.direction[a] = c.list("sourceDirection").at(a);
    p.momentPerLength = c.num("momentPerLength", p.momentPerLength);
    p.sourceSigmaM = c.num("sourceSigmaM", p.sourceSigmaM);
    p.sourceRadiusM = c.num("sourceRadiusM", p.sourceRadiusM);
    p.absorbing = c.num("absorbing", p.absorbing) != 0;
    p.spongeX = int(c.num("spongeX", p.spongeX));
    p.spongeZ = int(c.num("spongeZ", p.spongeZ));
    p.spongeStrength = c.num("spongeStrength", p.spongeStrength);
    p.absorber = c.num("absorber", 0) ? Absorber::CfsPml : Absorber::Sponge;
    p.cpml.targetReflection = c.num("cpmlReflection", p.cpml.targetReflection);
    p.cpml.kappaMax = c.num("cpmlKappaMax", p.cpml.kappaMax);
    p.cpml.frequency = c.num("cpmlFrequency", p.cpml.frequency);
    p.externalAbsorption = c.num("externalAbsorption", 0) != 0;
    p.receiverStart = int(c.num("receiverStart", p.receiverStart));
    p.receiverCount = int(c.num("receiverCount", p.receiverCount));
    p.receiverStride = int(c.num("receiverStride", p.receiverStride));
    p.receiverDepth = int(c.num("receiverDepth", p.receiverDepth));
    p.sampleIntervalMs = c.num("sampleIntervalMs", p.sampleIntervalMs);
    p.layered = c.num("layered", 0) != 0;
    p.attenuation.enabled = c.num("attenuation", 0) != 0;
    p.attenuation.mechanisms = int(c.num("mechanisms", p.attenuation.mechanisms));
    p.attenuation.minFrequency = c.num("qMinFrequency", p.attenuation.minFrequency);
    p.attenuation.maxFrequency = c.num("qMaxFrequency", p.attenuation.maxFrequency);
    p.attenuation.referenceFrequency = c.num("qReferenceFrequency", p.attenuation.referenceFrequency);
    p.attenuation.qp = c.num("qp", p.attenuation.qp);
    p.attenuation.qs = c.num("qs", p.attenuation.qs);
    p.importedSurface = c.num("importedSurface", 0) != 0;
    p.surfaceDatum = c.num("surfaceDatum", p.surfaceDatum);
    if (c.has("surface")) {
        const auto &s = c.list("surface");
        p.surfaceSamples.clear();
        for (std::size_t i = 0; i + 1 < s.size(); i += 2) p.surfaceSamples.push_back({s[i], s[i + 1]});
    }
    if (c.has("layers")) {
        // thickness vp vs density qp qs per layer
        const auto &l = c.list("layers");
        p.layers.clear();
        for (std::size_t i = 0; i + 6 <= l.size(); i += 6)
            p.layers.push_back({l[i], l[i + 1], l[i + 2], l[i + 3], l[i + 4], l[i + 5]});
    }
    return p;
}
void write(const std::filesystem::path &dir, const char *name, const double *v, std::size_t n) {
    std::ofstream out(dir / name, std::ios::binary);
    out.write(reinterpret_cast<const char *>(v), static_cast<std::streamsize>(n * sizeof(double)));
    if (!out) throw std::runtime_error(std::string("write failed: ") + name);
}
void write(const std::filesystem::path &dir, const char *name, const std::vector<double> &v) {
    write(dir, name, v.data(), v.size());
}
template <class A> std::vector<double> doubles(const A &a) { return a.toDouble(); }
} // namespace

int main(int argc, char **argv) {
    try {
        if (argc < 3) {
            std::cerr << "usage: ref2d case.txt outdir [steps] [threads] [dump_mesh] [warmup] [cpu|cuda]\n";
            return 2;
        }
        const Case c{readCase(argv[1])};
        const std::filesystem::path out(argv[2]);
        std::filesystem::create_directories(out);
        const int threads = argc > 4 ? std::atoi(argv[4]) : 1;
        const bool dumpMesh = argc > 5 ? std::atoi(argv[5]) != 0 : true;
        const auto p = parameters(c);
        Simulation sim;
        std::string error;
        const auto t0 = std::chrono::steady_clock::now();
        // backend: the reference's CPU loops, or its own CUDA engine (src/two_d/CudaEngine2D.cu) when
        // this driver is built with SEIS3D_HAS_CUDA
        const BackendKind3D kind = argc > 7 && std::string(argv[7]) == "cuda" ? BackendKind3D::Cuda : BackendKind3D::Cpu;
        if (!sim.initialize(p, error, kind, ComputeSettings3D{threads, -1})) {
            std::ofstream(out / "error.txt") << error << '\n';
            std::cerr << "initialize failed: " << error << '\n';
            return 3;
        }
        const double initMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        auto &s = *sim.impl_;
        const int steps = argc > 3 && std::atoi(argv[3]) >= 0 ? std::min(std::atoi(argv[3]), sim.totalSteps()) : sim.totalSteps();
        const std::size_t count = s.mesh.count;
        if (dumpMesh) {
            // Model arrays are converted to the session precision; promote to float64 for the dump.
            write(out, "metricA.bin", doubles(s.grid.metricA));
            write(out, "metricB.bin", doubles(s.grid.metricB));
            write(out, "jacobian.bin", doubles(s.grid.jacobian));
            write(out, "normals.bin", doubles(s.grid.normals));
            write(out, "coordinates.bin", doubles(s.grid.coordinates));
            write(out, "lambda.bin", doubles(s.lambda));
            write(out, "mu.bin", doubles(s.mu));
            write(out, "density.bin", doubles(s.grid.density));
            write(out, "vp.bin", doubles(s.grid.vp));
            write(out, "vs.bin", doubles(s.grid.vs));
            write(out, "source.bin", doubles(s.source));
            write(out, "damping.bin", doubles(s.damping));
            if (!s.sourceGradient[0].empty()) {
                write(out, "sourceGradientX.bin", doubles(s.sourceGradient[0]));
                write(out, "sourceGradientZ.bin", doubles(s.sourceGradient[1]));
            }
            if (!s.cpmlX.empty()) {
                write(out, "cpmlX.bin", doubles(s.cpmlX));
                write(out, "cpmlZ.bin", doubles(s.cpmlZ));
            }
            for (int l = 0; l < s.mesh.mechanisms; ++l) {
                const std::string p1 = "deltaP" + std::to_string(l) + ".bin", s1 = "deltaS" + std::to_string(l) + ".bin";
                write(out, p1.c_str(), doubles(s.deltaP[l]));
                write(out, s1.c_str(), doubles(s.deltaS[l]));
            }
        }
        // Optional untimed warm-up (benchmarks/ComputeBenchmark.cpp:71-75 times after warm-up).
        const int warmup = argc > 6 ? std::max(0, std::atoi(argv[6])) : 0;
        if (warmup > 0 && !sim.advance(warmup, error)) std::cerr << "warm-up failed: " << error << '\n';
        const auto t1 = std::chrono::steady_clock::now();
        if (steps > 0 && !sim.advance(steps, error)) {
            std::ofstream(out / "error.txt") << error << '\n';
            std::cerr << "advance failed: " << error << '\n';
        }
        const double runMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
        const auto snap = sim.snapshot(true);
        for (int f = 0; f < 5; ++f) write(out, ("field" + std::to_string(f) + ".bin").c_str(), snap.fields[f]);
        if (!snap.syy.empty()) write(out, "field5.bin", snap.syy);
        for (std::size_t m = 0; m < snap.memory.size(); ++m)
            write(out, ("field" + std::to_string(6 + m) + ".bin").c_str(), snap.memory[m]);
        if (!snap.boundaryMemory.empty()) write(out, "pml.bin", snap.boundaryMemory);
        // Raw per-step probe samples (the engine's own readback) and the resampled records.
        std::vector<double> vx, vz;
        for (const auto &r : sim.receivers()) {
            vx.insert(vx.end(), r.vx.begin(), r.vx.end());
            vz.insert(vz.end(), r.vz.begin(), r.vz.end());
        }
        write(out, "tracesVx.bin", vx);
        write(out, "tracesVz.bin", vz);
        const bool files = argc > 8 && std::string(argv[8]) == "files";
        if (files) { // the reference's receiver CSV (writeReceivers, CurvilinearSolver2D.cpp:811-855)
            std::string csvError;
            if (!writeReceivers(sim, out / "receivers.csv", csvError)) std::ofstream(out / "csv_error.txt") << csvError << '\n';
        }
        if (files) { // writeModelVts (src/two_d/ModelIo2D.cpp:75-145) with this run's compute settings
            std::string modelError;
            if (!writeModelVts(sim, out / "model.vts", ComputeSettings3D{threads, -1}, modelError))
                std::ofstream(out / "model_error.txt") << modelError << '\n';
        }
        if (files) { // writeSnapshot (CurvilinearSolver2D.cpp:725-810) with the default options and with every component
            std::string vtsError;
            SnapshotExportOptions all;
            all.components = {true, true, true, true, true, true, true};
            if (!writeSnapshot(sim, out / "snapshot.vts", vtsError, SnapshotExportOptions{}) ||
                !writeSnapshot(sim, out / "snapshot_all.vts", vtsError, all))
                std::ofstream(out / "vts_error.txt") << vtsError << '\n';
            // readProbes at a few logical nodes
            const auto &pp = sim.parameters();
            std::vector<std::array<int, 2>> nodes{{0, 0}, {pp.nx / 2, pp.nz / 3}, {pp.nx - 1, pp.nz - 1}, {pp.nx / 3, 0}};
            std::vector<std::array<double, 5>> probes;
            std::string probeError;
            if (sim.readProbes(nodes, probes, probeError)) {
                std::vector<double> flat;
                for (const auto &v : probes) flat.insert(flat.end(), v.begin(), v.end());
                write(out, "probes.bin", flat);
            }
        }
        if (files) { // the workbench's record view (src/two_d/ui/Workbench2D.cpp:251-268) through writeSegy
            SeisWave::RecordDataView data;
            data.dt = sim.recordDt();
            data.components = {"Vz", "Vx"};
            const auto &p = sim.parameters();
            const auto src = sim.grid().coordinates[sim.grid().modelIndex(p.sourceX < 0 ? p.nx / 2 : p.sourceX, p.sourceZ)];
            for (const auto &r : sim.receivers()) {
                SeisWave::TraceView t;
                t.position = {r.position[0], 0, r.position[1]};
                t.source = {src[0], 0, src[1]};
                t.channels[0] = r.vz;
                t.channels[1] = r.vx;
                data.traces.push_back(t);
            }
            std::string segyError;
            if (!SeisWave::writeSegy(data, 0, out / "vz_ieee32.sgy", segyError, false) ||
                !SeisWave::writeSegy(data, 1, out / "vx_ieee64.sgy", segyError, true))
                std::ofstream(out / "segy_error.txt") << segyError << '\n';
        }
        const auto &d = sim.diagnostics();
        std::ofstream meta(out / "meta.txt");
        meta.imbue(std::locale::classic());
        meta << std::setprecision(17);
        meta << "nx " << s.grid.nx << "\nnz " << s.grid.nz << "\ncount " << count << "\nh " << s.grid.h
             << "\nmodelOffsetX " << s.grid.modelOffsetX << "\ndt " << sim.dt() << "\nrecordDt " << sim.recordDt()
             << "\ntotal " << sim.totalSteps() << "\nsteps " << sim.step() << "\nfieldCount " << s.mesh.fieldCount
             << "\nmechanisms " << s.mesh.mechanisms << "\ncpmlCount " << d.cpmlScalars
             << "\ncpmlWidthX " << s.mesh.cpmlWidthX << "\ncpmlWidthZ " << s.mesh.cpmlWidthZ
             << "\nrates " << s.mesh.rates[0] << ' ' << s.mesh.rates[1] << ' ' << s.mesh.rates[2]
             << "\nsourceDirection " << s.mesh.sourceDirection[0] << ' ' << s.mesh.sourceDirection[1] << ' '
             << s.mesh.sourceDirection[2] << "\nsourceX " << s.p.sourceX << "\nsourceZ " << s.p.sourceZ
             << "\nreceivers " << sim.receivers().size() << "\nsamples "
             << (sim.receivers().empty() ? 0 : sim.receivers().front().vx.size()) << "\nprobeX";
        for (const auto &r : s.probes) meta << ' ' << r.x;
        meta << "\nprobeZ";
        for (const auto &r : s.probes) meta << ' ' << r.z;
        meta << "\nmaxMetric " << s.grid.maxMetric << "\nminJacobian " << s.grid.minJacobian << "\nmaxEdge "
             << s.grid.maxEdge << "\nflattenDepth " << s.grid.flattenDepth << "\nwaveDt " << d.waveDt
             << "\ndampingDt " << d.dampingDt << "\nsourceDt " << d.sourceDt << "\nrelaxationDt " << d.relaxationDt
             << "\ncpmlDt " << d.cpmlDt << "\nppw " << d.ppw << "\nenergy " << d.energy << "\npeakEnergy "
             << d.peakEnergy << "\nmaxVelocity " << d.maxVelocity << "\ntractionRelative " << d.tractionRelative
             << "\nfinite " << d.finite << "\nthreads " << s.threads << "\ninitMs " << initMs << "\nrunMs " << runMs
             << "\nmsPerStep " << (steps > 0 ? runMs / steps : 0.0) << "\nerror " << (error.empty() ? "none" : "set")
             << '\n';
        return 0;
    } catch (const std::exception &e) {
        std::cerr << "ref2d: " << e.what() << '\n';
        return 1;
    }
}

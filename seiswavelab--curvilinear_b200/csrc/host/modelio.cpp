// 2D model documents (include/swl_modelio.h): the reference's versioned ASCII VTS model schema of
// src/two_d/ModelIo2D.cpp, written from a session and read back into session parameters.
//
// The document is a VTK StructuredGrid of the logical model's nodes (x fastest, z positive down):
// field data with the schema version, every Parameters member, the GSLS / CFS-PML / precision /
// source-kernel settings, the layer and surface tables, the compute settings, the planned dt,
// record interval, step count and flattening depth, and an FNV-1a 64 checksum over all of it;
// point data Vp, Vs, Density, Jacobian, MetricA, MetricB and the node coordinates.  The field
// arrays appear in name order, as the reference's std::map keeps them.
#include "../../../include/swl_modelio.h"
#include "sessions.hpp"
#include <bit>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <locale>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace swl::modelio {
namespace {

using host::Failure;
using Arrays = std::map<std::string, std::vector<double>>;

void need(bool ok, const std::string &message) {
    if (!ok) throw std::runtime_error(message);
}

// FNV-1a, 64 bit, over the array names (NUL-terminated) and the values' little-endian IEEE bytes
// (a negative zero counted as zero).
struct Fnv1a {
    std::uint64_t h{14695981039346656037ULL};
    void byte(unsigned char b) { h = (h ^ b) * 1099511628211ULL; }
    void name(const std::string &s) {
        for (unsigned char c : s) byte(c);
        byte(0);
    }
    void number(double v) {
        const auto bits = std::bit_cast<std::uint64_t>(v == 0 ? 0.0 : v);
        for (int shift = 0; shift < 64; shift += 8) byte(static_cast<unsigned char>(bits >> shift));
    }
};

const char *const kPointArrays[6] = {"Vp", "Vs", "Density", "Jacobian", "MetricA", "MetricB"};
constexpr int kMaxAxisNodes = 16384, kMaxTimeSteps = 200000, kMaxSpongeCells = 512;

int componentsOf(const std::string &name) {
    if (name == "SourceDirection") return 3;
    if (name == "LayersThicknessVpVsDensity") return 4;
    if (name == "SurfaceSamplesXElevation" || name == "ModelChecksum") return 2;
    return 1;
}

// ModelIo2D.cpp:21-61: the document's field data (the schema version follows the newest feature used)
Arrays metadata(const host::Session2D &s, const swl_model_compute &c) {
    const auto &p = s.params;
    const auto &m = s.model;
    Arrays a;
    const auto add = [&](const char *name, double v) { a[name] = {v}; };
    const bool pml = p.absorber != 0 || p.cpmlReflection != 1e-4 || p.cpmlKappaMax != 3 || p.cpmlFrequency != 0;
    const bool fp32 = p.precision == SWL_FP32;
    const bool kernel = p.sourceSigmaM > 0;
    add("SeisWaveModel2DVersion", kernel ? 6 : fp32 ? 5 : p.externalAbsorption ? 4 : pml ? 3 : 2);
    if (fp32 || kernel) add("CalculationPrecision", p.precision);
    if (pml || p.externalAbsorption || fp32 || kernel)
        a["CfsPmlSettings"] = {double(p.absorber), p.cpmlReflection, p.cpmlKappaMax, p.cpmlFrequency};
    if (p.externalAbsorption || fp32 || kernel) add("ExternalAbsorption", p.externalAbsorption);
    if (kernel) a["PhysicalSourceKernelM"] = {p.sourceSigmaM, p.sourceRadiusM};
    const auto &q = p.attenuation;
    a["GSLSSettings"] = {double(q.enabled), double(q.mechanisms), q.minFrequency, q.maxFrequency, q.referenceFrequency, q.qp, q.qs};
    auto &layerQ = a["LayerQpQs"];
    for (const auto &l : p.layers) layerQ.insert(layerQ.end(), {l.qp, l.qs});
    add("Parameter_nx", p.nx), add("Parameter_nz", p.nz), add("Parameter_spacing", p.spacing), add("Parameter_vp", p.vp);
    add("Parameter_vs", p.vs), add("Parameter_density", p.density), add("Parameter_relief", p.relief);
    add("Parameter_wavelength", p.wavelength), add("Parameter_flattenDepth", p.flattenDepth), add("Parameter_frequency", p.frequency);
    add("Parameter_duration", p.duration), add("Parameter_cfl", p.cfl), add("Parameter_forcePerLength", p.forcePerLength);
    add("Parameter_momentPerLength", p.momentPerLength), add("Parameter_sourceX", p.sourceX), add("Parameter_sourceZ", p.sourceZ);
    add("Parameter_maxSteps", p.maxSteps), add("Parameter_absorbing", p.absorbing), add("Parameter_spongeX", p.spongeX);
    add("Parameter_spongeZ", p.spongeZ), add("Parameter_spongeStrength", p.spongeStrength);
    add("Parameter_receiverStart", p.receiverStart), add("Parameter_receiverCount", p.receiverCount);
    add("Parameter_receiverStride", p.receiverStride), add("Parameter_receiverDepth", p.receiverDepth);
    add("Parameter_sampleIntervalMs", p.sampleIntervalMs), add("Parameter_layered", p.layered);
    add("Parameter_importedSurface", p.importedSurface), add("Parameter_surfaceDatum", p.surfaceDatum);
    add("SourceKind", p.sourceKind);
    a["SourceDirection"] = {p.sourceDirection[0], p.sourceDirection[1], p.sourceDirection[2]};
    auto &layers = a["LayersThicknessVpVsDensity"];
    for (const auto &l : p.layers) layers.insert(layers.end(), {l.thickness, l.vp, l.vs, l.density});
    auto &surface = a["SurfaceSamplesXElevation"];
    for (const auto &v : p.surfaceSamples) surface.insert(surface.end(), {v[0], v[1]});
    add("BackendKind", c.backend), add("CpuThreadsRequested", c.cpu_threads), add("CudaDeviceRequested", c.cuda_device);
    add("ReferenceDtSeconds", m.dt), add("RecordIntervalSeconds", m.recordDt), add("EffectiveTotalSteps", m.total);
    add("EffectiveFlattenDepthM", m.flattenDepth), add("CoordinatesZPositiveDown", 1);
    return a;
}

double pointValue(const host::Model2D &m, int f, std::size_t n) {
    switch (f) {
    case 0: return m.vp[n];
    case 1: return m.vs[n];
    case 2: return m.density[n];
    case 3: return m.jacobian[n];
    case 4: return m.metricA[n];
    default: return m.metricB[n];
    }
}

// ---------------------------------------------------------------------- bounded VTS reading
std::string attribute(const std::string &tag, const std::string &name) {
    const auto at = tag.find(name + "=");
    need(at != std::string::npos, "Missing VTS attribute: " + name);
    const auto open = at + name.size() + 1;
    need(open < tag.size() && (tag[open] == '"' || tag[open] == '\''), "Invalid VTS attribute.");
    const auto close = tag.find(tag[open], open + 1);
    need(close != std::string::npos, "Unterminated VTS attribute.");
    return tag.substr(open + 1, close - open - 1);
}
std::string nextTag(std::istream &in) {
    in >> std::ws;
    need(in.get() == '<', "Expected VTS XML tag (truncated or unsupported file).");
    std::string t{"<"};
    for (int i = 0; i < 8192; ++i) {
        const auto c = in.get();
        need(c != std::char_traits<char>::eof(), "Truncated VTS XML tag.");
        t.push_back(static_cast<char>(c));
        if (c == '>') return t;
    }
    throw std::runtime_error("Oversized VTS XML tag.");
}
void expectTag(std::istream &in, const char *name) { need(nextTag(in) == name, std::string("Expected ") + name); }
int whole(double v, int lo, int hi) {
    need(std::isfinite(v) && v >= lo && v <= hi && v == std::floor(v), "Invalid integer model parameter.");
    return static_cast<int>(v);
}
// The `count` values of one array (and its closing tag), hashed when `hash` is set.
std::vector<double> readValues(std::istream &in, const std::string &header, Fnv1a *hash, std::size_t count, bool keep,
                               bool float32Allowed) {
    const bool f32 = attribute(header, "type") == "Float32";
    need(attribute(header, "format") == "ascii" && (attribute(header, "type") == "Float64" || (float32Allowed && f32)),
         "Model import requires supported SeisWave ASCII floating point VTS arrays.");
    const auto name = attribute(header, "Name");
    if (hash) hash->name(name);
    std::vector<double> values;
    if (keep) values.reserve(count);
    for (std::size_t n = 0; n < count; ++n) {
        double v{};
        need(static_cast<bool>(in >> v) && std::isfinite(v), "Missing or nonfinite VTS data: " + name);
        if (f32) {
            v = static_cast<float>(v);
            need(std::isfinite(v), "Float32 VTS value overflows: " + name);
        }
        if (hash) hash->number(v);
        if (keep) values.push_back(v);
    }
    expectTag(in, "</DataArray>");
    return values;
}

} // namespace

// writeModelVts (ModelIo2D.cpp:75-145)
void writeModel2D(const host::Session2D &s, const std::filesystem::path &path, const swl_model_compute &compute) {
    const auto &p = s.params;
    const auto &m = s.model;
    const char *pointType = p.precision == SWL_FP32 ? "Float32" : "Float64";
    Arrays arrays = metadata(s, compute);
    Fnv1a hash;
    for (const auto &[name, values] : arrays) {
        hash.name(name);
        for (double v : values) {
            need(std::isfinite(v), "Cannot save nonfinite model metadata.");
            hash.number(v);
        }
    }
    const auto eachNode = [&](auto &&visit) {
        for (int k = 0; k < p.nz; ++k)
            for (int i = 0; i < p.nx; ++i) visit(std::size_t(i + 3 + m.modelOffsetX) + std::size_t(m.nx) * std::size_t(k + 3));
    };
    for (int f = 0; f < 6; ++f) {
        hash.name(kPointArrays[f]);
        eachNode([&](std::size_t n) { hash.number(pointValue(m, f, n)); });
    }
    hash.name("Coordinates");
    eachNode([&](std::size_t n) {
        hash.number(m.coordinates[2 * n]);
        hash.number(0);
        hash.number(m.coordinates[2 * n + 1]);
    });
    arrays["ModelChecksum"] = {static_cast<double>(hash.h >> 32), static_cast<double>(hash.h & 0xffffffffULL)};

    std::filesystem::path pending = path;
    pending += ".partial";
    try {
        std::ofstream out(pending);
        need(static_cast<bool>(out), "Cannot create 2D model VTS file.");
        out.imbue(std::locale::classic());
        out << std::setprecision(17)
            << "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
            << "<StructuredGrid WholeExtent=\"0 " << p.nx - 1 << " 0 0 0 " << p.nz - 1 << "\">\n<FieldData>\n";
        for (const auto &[name, values] : arrays) {
            const int comps = componentsOf(name);
            out << "<DataArray type=\"Float64\" Name=\"" << name << "\" NumberOfComponents=\"" << comps << "\" NumberOfTuples=\""
                << values.size() / comps << "\" format=\"ascii\">";
            for (double v : values) out << v << ' ';
            out << "</DataArray>\n";
        }
        out << "</FieldData>\n<Piece Extent=\"0 " << p.nx - 1 << " 0 0 0 " << p.nz - 1 << "\"><PointData Scalars=\"Vp\">\n";
        for (int f = 0; f < 6; ++f) {
            out << "<DataArray type=\"" << pointType << "\" Name=\"" << kPointArrays[f] << "\" format=\"ascii\">\n";
            eachNode([&](std::size_t n) { out << pointValue(m, f, n) << ' '; });
            out << "\n</DataArray>\n";
        }
        out << "</PointData><Points><DataArray type=\"" << pointType << "\" Name=\"Coordinates\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        eachNode([&](std::size_t n) { out << m.coordinates[2 * n] << " 0 " << m.coordinates[2 * n + 1] << ' '; });
        out << "\n</DataArray></Points></Piece></StructuredGrid></VTKFile>\n";
        out.close();
        need(static_cast<bool>(out), "2D model VTS write failed.");
        std::filesystem::rename(pending, path); // an existing model survives a failed write
    } catch (...) {
        std::error_code ec;
        std::filesystem::remove(pending, ec);
        throw;
    }
}

struct Document2D {
    host::Params2D params;
    swl_model_compute compute{};
    double referenceDt{};
};

// readModelVts (ModelIo2D.cpp:146-255)
Document2D readModel2D(const std::filesystem::path &path) {
    std::ifstream in(path);
    in.imbue(std::locale::classic());
    need(static_cast<bool>(in), "Cannot open model VTS file.");
    auto head = nextTag(in);
    if (head.starts_with("<?xml")) head = nextTag(in);
    need(head.starts_with("<VTKFile ") && attribute(head, "type") == "StructuredGrid", "Expected a SeisWave 2D StructuredGrid model VTS.");
    const auto grid = nextTag(in);
    need(grid.starts_with("<StructuredGrid "), "Missing StructuredGrid.");
    expectTag(in, "<FieldData>");
    Arrays arrays;
    Fnv1a hash;
    for (;;) {
        const auto t = nextTag(in);
        if (t == "</FieldData>") break;
        need(t.starts_with("<DataArray ") && arrays.size() < 80, "Invalid model metadata.");
        const auto name = attribute(t, "Name");
        need(!arrays.contains(name), "Duplicate model metadata: " + name);
        const auto count = [&](const char *key, int hi) {
            const auto text = attribute(t, key);
            std::size_t end{};
            const double v = std::stod(text, &end);
            need(end == text.size(), "Invalid array size.");
            return whole(v, 0, hi);
        };
        const int comps = count("NumberOfComponents", 4), tuples = count("NumberOfTuples", 1000000);
        need(comps > 0 && std::size_t(comps) * tuples <= 2000000, "Oversized model metadata.");
        arrays[name] = readValues(in, t, name == "ModelChecksum" ? nullptr : &hash, std::size_t(comps) * tuples, true, false);
    }
    const auto one = [&](const char *key) {
        const auto it = arrays.find(key);
        need(it != arrays.end() && it->second.size() == 1, std::string("Missing model parameter: ") + key);
        return it->second[0];
    };
    const auto table = [&](const char *key) -> const std::vector<double> & {
        const auto it = arrays.find(key);
        if (it == arrays.end()) throw std::out_of_range("map::at");
        return it->second;
    };
    const int version = whole(one("SeisWaveModel2DVersion"), 1, 7);
    Document2D doc;
    auto &p = doc.params;
    const auto real = [&](const char *member, double &dst) { dst = one((std::string("Parameter_") + member).c_str()); };
    const auto integer = [&](const char *member, int &dst, int lo, int hi) {
        dst = whole(one((std::string("Parameter_") + member).c_str()), lo, hi);
    };
    integer("nx", p.nx, 8, kMaxAxisNodes), integer("nz", p.nz, 8, kMaxAxisNodes);
    real("spacing", p.spacing), real("vp", p.vp), real("vs", p.vs), real("density", p.density), real("relief", p.relief);
    real("wavelength", p.wavelength), real("flattenDepth", p.flattenDepth), real("frequency", p.frequency);
    real("duration", p.duration), real("cfl", p.cfl), real("forcePerLength", p.forcePerLength);
    real("momentPerLength", p.momentPerLength), integer("sourceX", p.sourceX, -1, p.nx - 1);
    integer("sourceZ", p.sourceZ, 0, p.nz - 1), integer("maxSteps", p.maxSteps, 0, kMaxTimeSteps);
    integer("spongeX", p.spongeX, 1, kMaxSpongeCells), integer("spongeZ", p.spongeZ, 1, kMaxSpongeCells);
    real("spongeStrength", p.spongeStrength), integer("receiverStart", p.receiverStart, 0, p.nx - 1);
    integer("receiverCount", p.receiverCount, 1, 1024), integer("receiverStride", p.receiverStride, 1, kMaxAxisNodes);
    integer("receiverDepth", p.receiverDepth, 0, p.nz - 1), real("sampleIntervalMs", p.sampleIntervalMs);
    real("surfaceDatum", p.surfaceDatum);
    p.absorbing = whole(one("Parameter_absorbing"), 0, 1) != 0;
    p.layered = whole(one("Parameter_layered"), 0, 1) != 0;
    p.importedSurface = whole(one("Parameter_importedSurface"), 0, 1) != 0;
    p.sourceKind = whole(one("SourceKind"), 0, 1);
    const auto &direction = table("SourceDirection");
    need(direction.size() == 3, "Invalid source direction.");
    for (int a = 0; a < 3; ++a) p.sourceDirection[a] = direction[a];
    if (version >= 6) {
        const auto &k = table("PhysicalSourceKernelM");
        need(k.size() == 2 && ((version >= 7 && k[0] == 0 && k[1] == 0) || (k[0] > 0 && k[1] >= k[0] && p.sourceKind == 0)),
             "Invalid physical source kernel metadata.");
        p.sourceSigmaM = k[0], p.sourceRadiusM = k[1];
    }
    if (version >= 7) {
        const auto &layout = table("SurfaceReceiverLayout");
        need(layout.size() == 2, "Invalid surface receiver policy.");
        whole(layout[1], 0, 1024);
        if (whole(layout[0], 0, 1) != 0 || layout[1] != 0)
            throw Failure(SWL_ERR_INVALID, "The automatic surface-receiver layout of this model file is not supported; "
                                           "save the model with an explicit receiver line.");
    }
    const auto &layers = table("LayersThicknessVpVsDensity");
    need(layers.size() % 4 == 0 && layers.size() <= 64, "Invalid model layer table.");
    p.layers.clear();
    for (std::size_t i = 0; i < layers.size(); i += 4) p.layers.push_back({layers[i], layers[i + 1], layers[i + 2], layers[i + 3], 100, 60});
    if (version >= 2) {
        const auto &q = table("GSLSSettings");
        need(q.size() == 7, "Invalid GSLS settings.");
        p.attenuation = {whole(q[0], 0, 1) != 0, whole(q[1], 1, 3), q[2], q[3], q[4], q[5], q[6]};
        host::validateGsls(p.attenuation);
        const auto &lq = table("LayerQpQs");
        need(lq.size() == 2 * p.layers.size(), "Layer Q table differs from material table.");
        for (std::size_t i = 0; i < p.layers.size(); ++i) p.layers[i].qp = lq[2 * i], p.layers[i].qs = lq[2 * i + 1];
    }
    if (version >= 5) p.precision = whole(one("CalculationPrecision"), 0, 1);
    if (version >= 4) p.externalAbsorption = whole(one("ExternalAbsorption"), 0, 1) != 0;
    if (version >= 3) {
        const auto &c = table("CfsPmlSettings");
        need(c.size() == 4, "Invalid CFS-PML metadata.");
        p.absorber = whole(c[0], 0, 1), p.cpmlReflection = c[1], p.cpmlKappaMax = c[2], p.cpmlFrequency = c[3];
        need(p.cpmlReflection >= 1e-8 && p.cpmlReflection <= .1 && p.cpmlKappaMax >= 1 && p.cpmlKappaMax <= 20 &&
                 p.cpmlFrequency >= 0 && p.cpmlFrequency <= 1e6,
             "Invalid CFS-PML profile settings.");
    }
    const auto &samples = table("SurfaceSamplesXElevation");
    need(samples.size() % 2 == 0, "Invalid model surface samples.");
    p.surfaceSamples.clear();
    for (std::size_t i = 0; i < samples.size(); i += 2) p.surfaceSamples.push_back({samples[i], samples[i + 1]});
    doc.compute.cpu_threads = whole(one("CpuThreadsRequested"), 0, 64);
    doc.compute.cuda_device = whole(one("CudaDeviceRequested"), -1, 100000);
    doc.compute.backend = whole(one("BackendKind"), 0, 1);
    doc.referenceDt = one("ReferenceDtSeconds");
    need(doc.referenceDt > 0 && one("CoordinatesZPositiveDown") == 1, "Invalid model time step / coordinate convention.");
    const std::string extent = "0 " + std::to_string(p.nx - 1) + " 0 0 0 " + std::to_string(p.nz - 1);
    need(attribute(grid, "WholeExtent") == extent, "Model dimensions disagree with VTS extent.");
    const auto piece = nextTag(in);
    need(piece.starts_with("<Piece ") && attribute(piece, "Extent") == extent, "Invalid model piece extent.");
    need(nextTag(in).starts_with("<PointData"), "Missing point material data.");
    const std::size_t count = std::size_t(p.nx) * p.nz;
    for (const char *name : kPointArrays) {
        const auto t = nextTag(in);
        need(t.starts_with("<DataArray ") && attribute(t, "Name") == name, "Missing model point array.");
        readValues(in, t, &hash, count, false, version >= 5);
    }
    expectTag(in, "</PointData>");
    expectTag(in, "<Points>");
    const auto coords = nextTag(in);
    need(attribute(coords, "Name") == "Coordinates" && attribute(coords, "NumberOfComponents") == "3", "Invalid model coordinates.");
    readValues(in, coords, &hash, count * 3, false, version >= 5);
    expectTag(in, "</Points>");
    expectTag(in, "</Piece>");
    expectTag(in, "</StructuredGrid>");
    expectTag(in, "</VTKFile>");
    in >> std::ws;
    need(in.peek() == std::char_traits<char>::eof(), "Unexpected trailing VTS content.");
    const auto &digest = table("ModelChecksum");
    need(digest.size() == 2 && digest[0] == static_cast<double>(hash.h >> 32) && digest[1] == static_cast<double>(hash.h & 0xffffffffULL),
         "Model checksum mismatch (file changed or damaged).");
    return doc;
}


// ------------------------------------------------------------------------------------- 3D
namespace {
constexpr int kMaxNodesPerAxis3D = 4096, kMaxSurfaceAxis3D = 4096;
constexpr std::size_t kMaxPaddedNodes3D = 306ull * 306 * 306, kMaxSurfaceSamples3D = 4000000;
const char *const kPointArrays3D[5] = {"Vp", "Vs", "Density", "LayerId", "Jacobian"};

// src/three_d/ModelIo3D.cpp:14-70
Arrays metadata3d(const host::Session3D &s, const swl_model_compute &c) {
    const auto &p = s.params;
    const auto &m = s.model;
    Arrays a;
    const auto add = [&](const char *name, double v) { a[name] = {v}; };
    add("SeisWaveModel3DVersion", p.surfaceGrid.empty() ? 1 : 2);
    add("NumericalSchemeVersion", 1);
    add("Parameter_nx", p.nx), add("Parameter_ny", p.ny), add("Parameter_nz", p.nz), add("Parameter_spacing", p.spacing);
    add("Parameter_vp", p.vp), add("Parameter_vs", p.vs), add("Parameter_density", p.density);
    add("Parameter_layeredMaterial", p.layered), add("Parameter_dominantFrequency", p.frequency);
    add("Parameter_sourceX", p.sourceX), add("Parameter_sourceY", p.sourceY), add("Parameter_sourceZ", p.sourceZ);
    add("Parameter_sourceForce", p.sourceForce), add("Parameter_sourceMoment", p.sourceMoment);
    add("Parameter_duration", p.duration), add("Parameter_maxSteps", p.maxSteps), add("Parameter_cflSafety", p.cfl);
    add("Parameter_topographyAmplitude", p.relief), add("Parameter_topographyWavelength", p.wavelength);
    add("Parameter_terrainTransitionDepth", p.flattenDepth);
    add("LayerDepthMode", p.layerDepthMode), add("SourceKind", p.sourceKind);
    a["SourceDirection"] = {p.sourceDirection[0], p.sourceDirection[1], p.sourceDirection[2]};
    auto &layers = a["LayersThicknessVpVsDensity"];
    auto &lengths = a["LayerNameLengths"];
    auto &names = a["LayerNamesUtf8"];
    for (std::size_t i = 0; i < p.layers.size(); ++i) {
        const auto &l = p.layers[i];
        layers.insert(layers.end(), {l.thickness, l.vp, l.vs, l.density});
        const std::string name = i < p.layerNames.size() ? p.layerNames[i] : std::string();
        lengths.push_back(double(name.size()));
        for (unsigned char ch : name) names.push_back(ch);
    }
    a["ReceiverArray"] = {double(p.receiverKind), double(p.receiverStartX), double(p.receiverStartY), double(p.receiverZ),
                          double(p.receiverCountX), double(p.receiverCountY), double(p.receiverStrideX), double(p.receiverStrideY)};
    a["AbsorbingBoundary"] = {p.absorbing ? 1. : 0., double(p.absorbingCells[0]), double(p.absorbingCells[1]),
                              double(p.absorbingCells[2]), p.absorbingStrength};
    add("BackendKind", c.backend), add("CpuThreadsRequested", c.cpu_threads), add("CudaDeviceRequested", c.cuda_device);
    add("ReferenceDtSeconds", m.dt), add("EffectiveTotalSteps", m.total), add("EffectiveFlattenDepthM", m.flattenDepth);
    add("CoordinatesZPositiveDown", 1);
    if (!p.surfaceGrid.empty()) {
        const auto &d = p.surfaceGrid;
        a["SurfaceGridGeometry"] = {double(d.nx), double(d.ny), d.spacing, d.originX, d.originY, d.datum};
        a["SurfaceGridElevations"] = d.elevations;
    }
    return a;
}
// materialLayerAtDepth3D(materialDepth3D) (include/Seis3D/MaterialModels3D.hpp:19-31) of padded node q
int layerOf(const host::Params3D &p, const host::Model3D &m, std::size_t q) {
    const std::size_t plane = std::size_t(m.nx) * m.ny;
    double depth;
    if (p.layerDepthMode == 0) depth = (static_cast<int>(q / plane) - 3) * p.spacing;
    else if (p.layerDepthMode == 2) depth = m.coordinates[3 * q + 2];
    else depth = m.coordinates[3 * q + 2] - m.coordinates[3 * (3 * plane + q % plane) + 2];
    double bottom = 0;
    for (std::size_t i = 0; i + 1 < p.layers.size(); ++i) {
        bottom += p.layers[i].thickness;
        if (depth < bottom) return static_cast<int>(i);
    }
    return static_cast<int>(p.layers.size()) - 1;
}
double pointValue3d(const host::Params3D &p, const host::Model3D &m, int f, std::size_t q) {
    if (f == 4) return m.jacobian[q];
    const int id = p.layered ? layerOf(p, m, q) : 0;
    if (f == 3) return id;
    if (p.layered) {
        const auto &l = p.layers[std::size_t(id)];
        return f == 0 ? l.vp : f == 1 ? l.vs : l.density;
    }
    return f == 0 ? p.vp : f == 1 ? p.vs : p.density;
}
} // namespace

// writeModelVts3D (src/three_d/ModelIo3D.cpp:87-170)
void writeModel3D(const host::Session3D &s, const std::filesystem::path &path, const swl_model_compute &compute) {
    const auto &p = s.params;
    const auto &m = s.model;
    Arrays arrays = metadata3d(s, compute);
    Fnv1a hash;
    for (const auto &[name, values] : arrays) {
        hash.name(name);
        for (double v : values) {
            need(std::isfinite(v), "Nonfinite model metadata.");
            hash.number(v);
        }
    }
    const auto eachNode = [&](auto &&visit) {
        for (int k = 0; k < p.nz; ++k)
            for (int j = 0; j < p.ny; ++j)
                for (int i = 0; i < p.nx; ++i)
                    visit(std::size_t(i + 3) + std::size_t(m.nx) * (std::size_t(j + 3) + std::size_t(m.ny) * std::size_t(k + 3)));
    };
    for (int f = 0; f < 5; ++f) {
        hash.name(kPointArrays3D[f]);
        eachNode([&](std::size_t q) { hash.number(pointValue3d(p, m, f, q)); });
    }
    hash.name("Coordinates");
    eachNode([&](std::size_t q) {
        for (int c = 0; c < 3; ++c) hash.number(m.coordinates[3 * q + c]);
    });
    arrays["ModelChecksum"] = {static_cast<double>(hash.h >> 32), static_cast<double>(hash.h & 0xffffffffULL)};
    if (!path.parent_path().empty()) std::filesystem::create_directories(path.parent_path());
    std::filesystem::path pending = path;
    pending += ".partial";
    try {
        std::ofstream out(pending);
        out.imbue(std::locale::classic());
        need(static_cast<bool>(out), "Cannot create 3D model VTS file.");
        out << std::setprecision(17) << "<?xml version=\"1.0\"?>\n<VTKFile type=\"StructuredGrid\" version=\"0.1\" "
                                         "byte_order=\"LittleEndian\">\n<StructuredGrid WholeExtent=\"0 "
            << p.nx - 1 << " 0 " << p.ny - 1 << " 0 " << p.nz - 1 << "\">\n<FieldData>\n";
        for (const auto &[name, values] : arrays) {
            const int comps = name == "SourceDirection" ? 3 : name == "LayersThicknessVpVsDensity" ? 4 : name == "ModelChecksum" ? 2 : 1;
            out << "<DataArray type=\"Float64\" Name=\"" << name << "\" NumberOfComponents=\"" << comps << "\" NumberOfTuples=\""
                << values.size() / comps << "\" format=\"ascii\">";
            for (double v : values) out << v << ' ';
            out << "</DataArray>\n";
        }
        out << "</FieldData><Piece Extent=\"0 " << p.nx - 1 << " 0 " << p.ny - 1 << " 0 " << p.nz - 1 << "\"><PointData Scalars=\"Vp\">\n";
        for (int f = 0; f < 5; ++f) {
            out << "<DataArray type=\"Float64\" Name=\"" << kPointArrays3D[f] << "\" format=\"ascii\">\n";
            eachNode([&](std::size_t q) { out << pointValue3d(p, m, f, q) << ' '; });
            out << "\n</DataArray>\n";
        }
        out << "</PointData><Points><DataArray type=\"Float64\" Name=\"Coordinates\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        eachNode([&](std::size_t q) {
            for (int c = 0; c < 3; ++c) out << m.coordinates[3 * q + c] << ' ';
        });
        out << "\n</DataArray></Points></Piece></StructuredGrid></VTKFile>\n";
        out.close();
        need(static_cast<bool>(out), "3D model VTS write failed.");
        std::filesystem::rename(pending, path);
    } catch (...) {
        std::error_code ec;
        std::filesystem::remove(pending, ec);
        throw;
    }
}

struct Document3D {
    host::Params3D params;
    swl_model_compute compute{};
    double referenceDt{};
};

// readModelVts3D (src/three_d/ModelIo3D.cpp:171-339)
Document3D readModel3D(const std::filesystem::path &path) {
    std::ifstream in(path);
    in.imbue(std::locale::classic());
    need(static_cast<bool>(in), "Cannot open 3D model VTS.");
    auto head = nextTag(in);
    if (head.starts_with("<?xml")) head = nextTag(in);
    need(head.starts_with("<VTKFile ") && attribute(head, "type") == "StructuredGrid", "Expected a 3D StructuredGrid model VTS.");
    const auto grid = nextTag(in);
    need(grid.starts_with("<StructuredGrid "), "Missing StructuredGrid.");
    expectTag(in, "<FieldData>");
    Arrays arrays;
    Fnv1a hash;
    for (;;) {
        const auto t = nextTag(in);
        if (t == "</FieldData>") break;
        need(t.starts_with("<DataArray ") && arrays.size() < 80, "Invalid model metadata.");
        const auto name = attribute(t, "Name");
        need(!arrays.contains(name), "Duplicate model metadata.");
        const auto count = [&](const char *key, int hi) {
            std::size_t end{};
            const auto text = attribute(t, key);
            const double v = std::stod(text, &end);
            need(end == text.size(), "Invalid metadata array size.");
            return whole(v, 0, hi);
        };
        const int limit = name == "SurfaceGridElevations" ? static_cast<int>(kMaxSurfaceSamples3D) : 65536;
        const int comps = count("NumberOfComponents", 4), tuples = count("NumberOfTuples", limit);
        need(comps > 0 && std::size_t(comps) * tuples <= std::size_t(limit), "Oversized model metadata.");
        arrays[name] = readValues(in, t, name == "ModelChecksum" ? nullptr : &hash, std::size_t(comps) * tuples, true, false);
    }
    const auto one = [&](const char *key) {
        const auto it = arrays.find(key);
        need(it != arrays.end() && it->second.size() == 1, std::string("Missing model parameter: ") + key);
        return it->second[0];
    };
    const auto table = [&](const char *key) -> std::vector<double> & {
        const auto it = arrays.find(key);
        if (it == arrays.end()) throw std::out_of_range("map::at");
        return it->second;
    };
    const int version = whole(one("SeisWaveModel3DVersion"), 1, 2);
    need(one("NumericalSchemeVersion") == 1, "Unsupported 3D model schema or numerical scheme.");
    Document3D doc;
    auto &p = doc.params;
    const auto real = [&](const char *member, double &dst) { dst = one((std::string("Parameter_") + member).c_str()); };
    const auto integer = [&](const char *member, int &dst, int lo, int hi) {
        dst = whole(one((std::string("Parameter_") + member).c_str()), lo, hi);
    };
    integer("nx", p.nx, 8, kMaxNodesPerAxis3D), integer("ny", p.ny, 8, kMaxNodesPerAxis3D), integer("nz", p.nz, 8, kMaxNodesPerAxis3D);
    need(std::size_t(p.nx + 6) * (p.ny + 6) * (p.nz + 6) <= kMaxPaddedNodes3D, "Model exceeds the total padded-node budget.");
    real("spacing", p.spacing), real("vp", p.vp), real("vs", p.vs), real("density", p.density);
    real("dominantFrequency", p.frequency);
    integer("sourceX", p.sourceX, -1, p.nx - 1), integer("sourceY", p.sourceY, -1, p.ny - 1), integer("sourceZ", p.sourceZ, 0, p.nz - 1);
    real("sourceForce", p.sourceForce), real("sourceMoment", p.sourceMoment), real("duration", p.duration);
    integer("maxSteps", p.maxSteps, 0, 20000);
    real("cflSafety", p.cfl), real("topographyAmplitude", p.relief), real("topographyWavelength", p.wavelength);
    real("terrainTransitionDepth", p.flattenDepth);
    p.layered = whole(one("Parameter_layeredMaterial"), 0, 1) != 0;
    p.layerDepthMode = whole(one("LayerDepthMode"), 0, 2);
    p.sourceKind = whole(one("SourceKind"), 0, 1);
    const auto &direction = table("SourceDirection");
    need(direction.size() == 3, "Invalid source direction.");
    for (int a = 0; a < 3; ++a) p.sourceDirection[a] = direction[a];
    const auto &layers = table("LayersThicknessVpVsDensity");
    const auto &lengths = table("LayerNameLengths");
    const auto &names = table("LayerNamesUtf8");
    need(layers.size() % 4 == 0 && layers.size() <= 32 && lengths.size() == layers.size() / 4, "Invalid layer table.");
    std::size_t cursor = 0;
    p.layers.clear();
    for (std::size_t i = 0; i < lengths.size(); ++i) {
        const auto n = static_cast<std::size_t>(whole(lengths[i], 0, 8192));
        need(n <= names.size() - cursor, "Invalid UTF8 layer-name length.");
        std::string name;
        for (std::size_t c = 0; c < n; ++c) name.push_back(static_cast<char>(whole(names[cursor++], 0, 255)));
        p.layers.push_back({layers[4 * i], layers[4 * i + 1], layers[4 * i + 2], layers[4 * i + 3]});
        p.layerNames.push_back(name);
    }
    need(cursor == names.size(), "Unused layer-name bytes.");
    const auto &r = table("ReceiverArray");
    need(r.size() == 8, "Invalid receiver array.");
    p.receiverKind = whole(r[0], 0, 3), p.receiverStartX = whole(r[1], -1, p.nx - 1), p.receiverStartY = whole(r[2], -1, p.ny - 1);
    p.receiverZ = whole(r[3], 0, p.nz - 1), p.receiverCountX = whole(r[4], 1, 1024), p.receiverCountY = whole(r[5], 1, 1024);
    p.receiverStrideX = whole(r[6], 1, kMaxNodesPerAxis3D), p.receiverStrideY = whole(r[7], 1, kMaxNodesPerAxis3D);
    const auto &b = table("AbsorbingBoundary");
    need(b.size() == 5, "Invalid absorbing settings.");
    p.absorbing = whole(b[0], 0, 1) != 0;
    p.absorbingCells = {whole(b[1], 1, 64), whole(b[2], 1, 64), whole(b[3], 1, 64)};
    p.absorbingStrength = b[4];
    doc.compute.backend = whole(one("BackendKind"), 0, 1);
    doc.compute.cpu_threads = whole(one("CpuThreadsRequested"), 0, 64);
    doc.compute.cuda_device = whole(one("CudaDeviceRequested"), -1, 100000);
    doc.referenceDt = one("ReferenceDtSeconds");
    need(doc.referenceDt > 0 && one("CoordinatesZPositiveDown") == 1, "Invalid model conventions.");
    if (version == 2) {
        const auto &g = table("SurfaceGridGeometry");
        need(g.size() == 6, "Invalid embedded DEM geometry.");
        auto &dem = p.surfaceGrid;
        dem.nx = whole(g[0], 2, kMaxSurfaceAxis3D), dem.ny = whole(g[1], 2, kMaxSurfaceAxis3D);
        dem.spacing = g[2], dem.originX = g[3], dem.originY = g[4], dem.datum = g[5];
        dem.elevations = std::move(table("SurfaceGridElevations"));
        // SurfaceGrid3D::validate (src/three_d/SurfaceGrid3D.cpp:8-17)
        need(std::size_t(dem.nx) * dem.ny <= kMaxSurfaceSamples3D && dem.elevations.size() == std::size_t(dem.nx) * dem.ny &&
                 std::isfinite(dem.spacing) && dem.spacing > 0 && std::isfinite(dem.originX) && std::isfinite(dem.originY) &&
                 std::isfinite(dem.datum) && std::isfinite((dem.nx - 1) * dem.spacing) && std::isfinite((dem.ny - 1) * dem.spacing),
             "DEM array requires 2..4096 rows/columns, at most 4 million samples, positive metre spacing and finite origin/datum.");
        for (double h : dem.elevations) need(std::isfinite(h) && std::fabs(h) <= 1e7, "DEM contains missing, nonfinite or unreasonable elevations.");
    } else {
        need(!arrays.contains("SurfaceGridGeometry") && !arrays.contains("SurfaceGridElevations"), "DEM metadata requires model schema 2.");
    }
    const std::string extent = "0 " + std::to_string(p.nx - 1) + " 0 " + std::to_string(p.ny - 1) + " 0 " + std::to_string(p.nz - 1);
    need(attribute(grid, "WholeExtent") == extent, "Model/grid extent mismatch.");
    const auto piece = nextTag(in);
    need(piece.starts_with("<Piece ") && attribute(piece, "Extent") == extent, "Invalid piece extent.");
    need(nextTag(in).starts_with("<PointData"), "Missing model arrays.");
    const std::size_t count = std::size_t(p.nx) * p.ny * p.nz;
    for (const char *name : kPointArrays3D) {
        const auto t = nextTag(in);
        need(t.starts_with("<DataArray ") && attribute(t, "Name") == name, "Missing model point array.");
        readValues(in, t, &hash, count, false, false);
    }
    expectTag(in, "</PointData>");
    expectTag(in, "<Points>");
    const auto coords = nextTag(in);
    need(attribute(coords, "Name") == "Coordinates" && attribute(coords, "NumberOfComponents") == "3", "Invalid model coordinates.");
    readValues(in, coords, &hash, count * 3, false, false);
    expectTag(in, "</Points>");
    expectTag(in, "</Piece>");
    expectTag(in, "</StructuredGrid>");
    expectTag(in, "</VTKFile>");
    in >> std::ws;
    need(in.peek() == std::char_traits<char>::eof(), "Trailing model data.");
    const auto &digest = table("ModelChecksum");
    need(digest.size() == 2 && digest[0] == static_cast<double>(hash.h >> 32) && digest[1] == static_cast<double>(hash.h & 0xffffffffULL),
         "Model checksum mismatch.");
    return doc;
}

} // namespace swl::modelio

// ------------------------------------------------------------------------------------ C ABI
struct swl2d_model_document {
    swl::modelio::Document2D doc;
    std::vector<swl_layer2d> layers;
    std::vector<double> surface;
};

extern "C" {
swl_status swl2d_session_write_model(const swl2d_session *s, const char *path, const swl_model_compute *compute) {
    return swl::host::guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "Initialize the 2D model before saving.");
        if (!path || !compute) throw swl::host::Failure(SWL_ERR_INVALID, "path and compute settings are required");
        swl::modelio::writeModel2D(*s, path, *compute);
    });
}
swl_status swl2d_read_model(const char *path, swl2d_model_document **out) {
    return swl::host::guard([&] {
        if (!path || !out) throw swl::host::Failure(SWL_ERR_INVALID, "path and out are required");
        *out = nullptr;
        auto d = std::make_unique<swl2d_model_document>();
        d->doc = swl::modelio::readModel2D(path);
        for (const auto &l : d->doc.params.layers) d->layers.push_back({l.thickness, l.vp, l.vs, l.density, l.qp, l.qs});
        for (const auto &v : d->doc.params.surfaceSamples) d->surface.insert(d->surface.end(), {v[0], v[1]});
        *out = d.release();
    });
}
swl_status swl2d_model_document_params(const swl2d_model_document *d, swl_params2d *c, swl_model_compute *compute, double *reference_dt) {
    return swl::host::guard([&] {
        if (!d || !c) throw swl::host::Failure(SWL_ERR_INVALID, "document and params are required");
        const auto &p = d->doc.params;
        swl2d_params_default(c);
        c->precision = p.precision, c->nx = p.nx, c->nz = p.nz;
        c->spacing = p.spacing, c->vp = p.vp, c->vs = p.vs, c->density = p.density, c->relief = p.relief, c->wavelength = p.wavelength;
        c->flatten_depth = p.flattenDepth, c->frequency = p.frequency, c->duration = p.duration, c->cfl = p.cfl;
        c->force_per_length = p.forcePerLength, c->source_x = p.sourceX, c->source_z = p.sourceZ, c->max_steps = p.maxSteps;
        c->source_kind = p.sourceKind;
        for (int a = 0; a < 3; ++a) c->source_direction[a] = p.sourceDirection[a];
        c->moment_per_length = p.momentPerLength, c->source_sigma_m = p.sourceSigmaM, c->source_radius_m = p.sourceRadiusM;
        c->absorbing = p.absorbing, c->sponge_x = p.spongeX, c->sponge_z = p.spongeZ, c->sponge_strength = p.spongeStrength;
        c->absorber = p.absorber, c->cpml_reflection = p.cpmlReflection, c->cpml_kappa_max = p.cpmlKappaMax;
        c->cpml_frequency = p.cpmlFrequency, c->external_absorption = p.externalAbsorption;
        c->receiver_start = p.receiverStart, c->receiver_count = p.receiverCount, c->receiver_stride = p.receiverStride;
        c->receiver_depth = p.receiverDepth, c->sample_interval_ms = p.sampleIntervalMs;
        c->layered = p.layered, c->n_layers = int32_t(d->layers.size()), c->layers = d->layers.data();
        c->attenuation = p.attenuation.enabled, c->mechanisms = p.attenuation.mechanisms;
        c->q_min_frequency = p.attenuation.minFrequency, c->q_max_frequency = p.attenuation.maxFrequency;
        c->q_reference_frequency = p.attenuation.referenceFrequency, c->qp = p.attenuation.qp, c->qs = p.attenuation.qs;
        c->imported_surface = p.importedSurface, c->surface_datum = p.surfaceDatum;
        c->n_surface = int32_t(d->surface.size() / 2), c->surface_xz = d->surface.empty() ? nullptr : d->surface.data();
        if (compute) *compute = d->doc.compute;
        if (reference_dt) *reference_dt = d->doc.referenceDt;
    });
}
void swl2d_model_document_free(swl2d_model_document *d) { delete d; }
} // extern "C"

struct swl3d_model_document {
    swl::modelio::Document3D doc;
    std::vector<swl_layer3d> layers;
    std::vector<const char *> names;
};

extern "C" {
swl_status swl3d_session_write_model(const swl3d_session *s, const char *path, const swl_model_compute *compute) {
    return swl::host::guard([&] {
        if (!s) throw swl::host::Failure(SWL_ERR_INVALID, "Initialize the 3D model before saving.");
        if (!path || !compute) throw swl::host::Failure(SWL_ERR_INVALID, "path and compute settings are required");
        swl::modelio::writeModel3D(*s, path, *compute);
    });
}
swl_status swl3d_read_model(const char *path, swl3d_model_document **out) {
    return swl::host::guard([&] {
        if (!path || !out) throw swl::host::Failure(SWL_ERR_INVALID, "path and out are required");
        *out = nullptr;
        auto d = std::make_unique<swl3d_model_document>();
        d->doc = swl::modelio::readModel3D(path);
        for (const auto &l : d->doc.params.layers) d->layers.push_back({l.thickness, l.vp, l.vs, l.density});
        for (const auto &n : d->doc.params.layerNames) d->names.push_back(n.c_str());
        *out = d.release();
    });
}
swl_status swl3d_model_document_params(const swl3d_model_document *d, swl_params3d *c, swl_model_compute *compute, double *reference_dt) {
    return swl::host::guard([&] {
        if (!d || !c) throw swl::host::Failure(SWL_ERR_INVALID, "document and params are required");
        const auto &p = d->doc.params;
        swl3d_params_default(c);
        c->precision = p.precision, c->nx = p.nx, c->ny = p.ny, c->nz = p.nz;
        c->spacing = p.spacing, c->vp = p.vp, c->vs = p.vs, c->density = p.density;
        c->layered = p.layered, c->layer_depth_mode = p.layerDepthMode;
        c->n_layers = int32_t(d->layers.size()), c->layers = d->layers.data();
        c->layer_names = d->names.empty() ? nullptr : d->names.data();
        c->frequency = p.frequency, c->source_x = p.sourceX, c->source_y = p.sourceY, c->source_z = p.sourceZ;
        c->source_kind = p.sourceKind;
        for (int a = 0; a < 3; ++a) c->source_direction[a] = p.sourceDirection[a];
        c->source_force = p.sourceForce, c->source_moment = p.sourceMoment, c->duration = p.duration, c->max_steps = p.maxSteps;
        c->cfl = p.cfl, c->relief = p.relief, c->wavelength = p.wavelength, c->flatten_depth = p.flattenDepth;
        if (!p.surfaceGrid.empty()) {
            const auto &g = p.surfaceGrid;
            c->dem_nx = g.nx, c->dem_ny = g.ny, c->dem_spacing = g.spacing, c->dem_origin_x = g.originX;
            c->dem_origin_y = g.originY, c->dem_datum = g.datum, c->dem_elevations = g.elevations.data();
        }
        c->receiver_kind = p.receiverKind, c->receiver_start_x = p.receiverStartX, c->receiver_start_y = p.receiverStartY;
        c->receiver_z = p.receiverZ, c->receiver_count_x = p.receiverCountX, c->receiver_count_y = p.receiverCountY;
        c->receiver_stride_x = p.receiverStrideX, c->receiver_stride_y = p.receiverStrideY;
        c->absorbing = p.absorbing;
        for (int a = 0; a < 3; ++a) c->absorbing_cells[a] = p.absorbingCells[a];
        c->absorbing_strength = p.absorbingStrength;
        if (compute) *compute = d->doc.compute;
        if (reference_dt) *reference_dt = d->doc.referenceDt;
    });
}
void swl3d_model_document_free(swl3d_model_document *d) { delete d; }
} // extern "C"

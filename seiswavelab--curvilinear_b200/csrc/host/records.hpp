// Receiver record sets and their SEG-Y encoding (the file format of src/common/SegyIo.cpp).
#pragma once
#include <array>
#include <cstddef>
#include <filesystem>
#include <string>
#include <vector>

namespace swl::records {

// One trace of a record set: geometry plus one sample array per component (not owned).
struct Trace {
    std::array<double, 3> position{}, source{};
    double start{};
    std::array<const double *, 3> channel{};
};
struct RecordSet {
    std::vector<Trace> traces;
    std::vector<std::string> components;
    std::size_t samples{};
    double dt{};
    std::string units{"m/s"};
};
// SegyExportProfile order: exact IEEE32, exact IEEE64, legacy IBM32, compatible IEEE32.
struct SegyOptions {
    int profile{0};
    double gain{1};
    double interval{0}; // seconds; 0 keeps dt
};
// Throws std::runtime_error with the reference's message; a failed export leaves `path` as it was.
void writeSegy(const RecordSet &records, int component, const std::filesystem::path &path, const SegyOptions &options);

struct ImportedTrace {
    std::array<double, 3> position{}, source{};
    double start{};
    std::vector<double> samples;
};
struct Imported {
    double dt{};
    std::string component{"Amplitude"}, units{"raw"}, description;
    std::vector<ImportedTrace> traces;
};
Imported readSegy(const std::filesystem::path &path);

} // namespace swl::records

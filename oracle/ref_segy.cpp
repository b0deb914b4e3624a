// Test infrastructure only: drives the reference's own SEG-Y writer and reader
// (src/common/SegyIo.cpp, compiled from its sources by oracle/Makefile) so that the record
// output of this library can be compared byte for byte.  Nothing in the product links or runs
// this program.
//
// Usage:
//   ref_segy write <records.txt> <component> <profile 0-3> <gain> <interval_s> <out.sgy>
//   ref_segy read  <in.sgy> <dump.txt>
// records.txt (classic locale, values written with 17 significant digits):
//   dt <s>
//   units <text>
//   components <n> <name>...
//   traces <n> <samples>
//   then per trace: px py pz sx sy sz start, followed by <n components> lines of samples
// dump.txt: "ok" or "error <message>", then dt, component, units, description and per trace
// position, source, start and samples.
#include "SeisCommon/SegyIo.hpp"
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <locale>
#include <sstream>
#include <string>
#include <vector>

namespace {
int writeCmd(char **argv) {
    std::ifstream in(argv[2]);
    in.imbue(std::locale::classic());
    std::string key;
    double dt = 0;
    std::string units;
    int nc = 0;
    std::vector<std::string> names;
    std::size_t nt = 0, ns = 0;
    in >> key >> dt >> key >> units >> key >> nc;
    names.resize(nc);
    for (auto &n : names) in >> n;
    in >> key >> nt >> ns;
    std::vector<std::vector<std::vector<double>>> data(nt, std::vector<std::vector<double>>(nc, std::vector<double>(ns)));
    SeisWave::RecordDataView view;
    view.dt = dt;
    view.units = units;
    view.components = names;
    for (std::size_t r = 0; r < nt; ++r) {
        SeisWave::TraceView t;
        for (auto &v : t.position) in >> v;
        for (auto &v : t.source) in >> v;
        in >> t.startTime;
        for (int c = 0; c < nc; ++c)
            for (auto &v : data[r][c]) in >> v;
        for (int c = 0; c < nc; ++c) t.channels[c] = data[r][c];
        view.traces.push_back(t);
    }
    if (!in) {
        std::cerr << "bad records file\n";
        return 2;
    }
    SeisWave::SegyExportOptions options;
    options.profile = static_cast<SeisWave::SegyExportProfile>(std::stoi(argv[4]));
    options.sampleGain = std::stod(argv[5]);
    options.sampleIntervalSeconds = std::stod(argv[6]);
    std::string error;
    const bool ok = SeisWave::writeSegy(view, std::stoi(argv[3]), argv[7], error, options);
    std::cout << (ok ? "ok" : "error " + error) << '\n';
    return 0;
}
int readCmd(char **argv) {
    SeisWave::ImportedRecords records;
    std::string error;
    const bool ok = SeisWave::readSegy(argv[2], records, error);
    std::ofstream out(argv[3]);
    out.imbue(std::locale::classic());
    out << std::setprecision(17);
    if (!ok) {
        out << "error " << error << '\n';
        return 0;
    }
    out << "ok\n" << records.dt << '\n' << records.component << '\n' << records.units << '\n' << records.description << '\n';
    out << records.traces.size() << '\n';
    for (const auto &t : records.traces) {
        for (double v : t.position) out << v << ' ';
        for (double v : t.source) out << v << ' ';
        out << t.startTime << ' ' << t.samples.size() << '\n';
        for (double v : t.samples) out << v << ' ';
        out << '\n';
    }
    return 0;
}
} // namespace

int main(int argc, char **argv) {
    if (argc == 8 && std::string(argv[1]) == "write") return writeCmd(argv);
    if (argc == 4 && std::string(argv[1]) == "read") return readCmd(argv);
    std::cerr << "usage: ref_segy write <records.txt> <component> <profile> <gain> <interval_s> <out.sgy>\n"
                 "       ref_segy read <in.sgy> <dump.txt>\n";
    return 2;
}

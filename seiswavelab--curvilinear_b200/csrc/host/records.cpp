// SEG-Y export and import of receiver records, and their C ABI (include/swl_records.h).
//
// The layout is the one src/common/SegyIo.cpp writes and reads, so the files are exchangeable
// with the reference and with its downstream tools:
//   - 3200-byte textual header (ASCII, or EBCDIC code page 037 for the legacy IBM profile), with
//     the exact dt, units, multiplier, output peak and underflow count on lines 1-13 and 40;
//   - 400-byte binary header, big endian: rev 2 (exact IEEE64 microsecond interval at 3273-3280,
//     byte-order marker, trace count and header offset) or rev 1 for the compatible profiles;
//   - per trace a 240-byte header (sequence numbers, trace id 12 = Vz / 14 = Vx, signed offset,
//     coordinates and elevations in millimetres with scalar -1000, delay, sample count and
//     interval, midpoint, units code) followed by IEEE32, IEEE64 or IBM32 samples.
// The importer accepts rev 0-2 files with fixed 240-byte trace headers in sample formats 1, 2,
// 3, 5, 6 and 8, in either byte order.
#include "records.hpp"
#include "../../../include/swl_records.h"
#include "../runtime.cuh"
#include <algorithm>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <memory>
#include <sstream>
#include <stdexcept>

namespace swl::records {
namespace {

using Bytes = std::vector<unsigned char>;

void expect(bool condition, const char *message) {
    if (!condition) throw std::runtime_error(message);
}

// Big-endian field writer over a fixed block.
struct Block {
    Bytes bytes;
    explicit Block(std::size_t n, unsigned char fill = 0) : bytes(n, fill) {}
    void put(std::size_t at, std::uint64_t value, int width) {
        for (int i = width - 1; i >= 0; --i, value >>= 8) bytes[at + i] = static_cast<unsigned char>(value & 0xff);
    }
    void i32(std::size_t at, std::int32_t v) { put(at, static_cast<std::uint32_t>(v), 4); }
};

// Unsigned field reader in either byte order.
struct Fields {
    const Bytes &b;
    bool little;
    std::uint64_t u(std::size_t at, int width) const {
        std::uint64_t v = 0;
        for (int i = 0; i < width; ++i) v = (v << 8) | b[at + (little ? width - 1 - i : i)];
        return v;
    }
    std::int16_t s16(std::size_t at) const { return std::bit_cast<std::int16_t>(static_cast<std::uint16_t>(u(at, 2))); }
    std::int32_t s32(std::size_t at) const { return std::bit_cast<std::int32_t>(static_cast<std::uint32_t>(u(at, 4))); }
    double f64(std::size_t at) const { return std::bit_cast<double>(u(at, 8)); }
};

// IBM code page 037 for ASCII 0-127.
constexpr unsigned char kCp037[128] = {
    0x00, 0x01, 0x02, 0x03, 0x37, 0x2d, 0x2e, 0x2f, 0x16, 0x05, 0x25, 0x0b, 0x0c, 0x0d, 0x0e, 0x0f,
    0x10, 0x11, 0x12, 0x13, 0x3c, 0x3d, 0x32, 0x26, 0x18, 0x19, 0x3f, 0x27, 0x1c, 0x1d, 0x1e, 0x1f,
    0x40, 0x5a, 0x7f, 0x7b, 0x5b, 0x6c, 0x50, 0x7d, 0x4d, 0x5d, 0x5c, 0x4e, 0x6b, 0x60, 0x4b, 0x61,
    0xf0, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0x7a, 0x5e, 0x4c, 0x7e, 0x6e, 0x6f,
    0x7c, 0xc1, 0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xd1, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6,
    0xd7, 0xd8, 0xd9, 0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xba, 0xe0, 0xbb, 0xb0, 0x6d,
    0x79, 0x81, 0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x91, 0x92, 0x93, 0x94, 0x95, 0x96,
    0x97, 0x98, 0x99, 0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xc0, 0x4f, 0xd0, 0xa1, 0x07,
};

// IBM System/360 single precision: sign, excess-64 base-16 exponent, 24-bit fraction 0.F,
// rounded to nearest (ties away from zero); values below the smallest normalised number are 0.
std::uint32_t toIbm32(double v) {
    if (v == 0) return 0;
    const double mag = std::fabs(v);
    int binary = 0;
    std::frexp(mag, &binary);                                  // mag = m 2^binary, m in [0.5, 1)
    int hex = static_cast<int>(std::ceil(binary / 4.0));        // mag < 16^hex
    if (hex < -64) return 0;
    expect(hex <= 63, "SEG-Y IBM32 sample overflow; reduce the export multiplier.");
    auto fraction = static_cast<std::uint32_t>(std::llround(std::ldexp(mag, 24 - 4 * hex)));
    if (fraction == (1u << 24)) fraction = 1u << 20, ++hex; // rounding carried into a new digit
    expect(hex <= 63, "SEG-Y IBM32 rounding overflow.");
    return (std::signbit(v) ? 0x80000000u : 0u) | (static_cast<std::uint32_t>(hex + 64) << 24) | fraction;
}
double fromIbm32(std::uint32_t bits) {
    const std::uint32_t fraction = bits & 0xffffff;
    double v = fraction ? std::ldexp(static_cast<double>(fraction), 4 * (static_cast<int>((bits >> 24) & 0x7f) - 64) - 24) : 0.0;
    return (bits & 0x80000000u) ? -v : v;
}

std::int32_t toMillimetres(double metres) {
    expect(std::isfinite(metres) && std::fabs(metres * 1000) < std::numeric_limits<std::int32_t>::max(),
           "SEG-Y coordinates exceed the supported millimetre range.");
    return static_cast<std::int32_t>(std::llround(metres * 1000));
}
std::string exact(double v) {
    std::ostringstream s;
    s << std::setprecision(17) << v;
    return s.str();
}
int bytesPerSample(int format) {
    switch (format) {
    case 1: case 2: case 5: return 4;
    case 3: return 2;
    case 6: return 8;
    case 8: return 1;
    default: return 0;
    }
}
double headerScale(std::int16_t s) { return s > 0 ? s : s < 0 ? -1.0 / s : 1.0; }

void writeAll(std::ofstream &out, const Bytes &b) {
    out.write(reinterpret_cast<const char *>(b.data()), static_cast<std::streamsize>(b.size()));
    expect(static_cast<bool>(out), "SEG-Y write failed.");
}

} // namespace

void writeSegy(const RecordSet &rec, int component, const std::filesystem::path &path, const SegyOptions &o) {
    std::filesystem::path partial;
    try {
        const bool ieee64 = o.profile == SWL_SEGY_IEEE64, ibm = o.profile == SWL_SEGY_IBM32;
        const bool legacy = ibm || o.profile == SWL_SEGY_COMPATIBLE_IEEE32; // rev 1, whole-microsecond dt
        expect(o.profile >= SWL_SEGY_IEEE32 && o.profile <= SWL_SEGY_COMPATIBLE_IEEE32, "Unknown SEG-Y export profile.");
        expect(std::isfinite(o.gain) && o.gain > 0, "SEG-Y export multiplier must be finite and positive.");
        expect(std::isfinite(o.interval) && o.interval >= 0, "Invalid SEG-Y output sampling interval.");
        expect(!rec.traces.empty() && component >= 0 && component < static_cast<int>(rec.components.size()),
               "Select an existing raw component before SEG-Y export.");
        expect(std::isfinite(rec.dt) && rec.dt > 0, "Invalid source sampling interval.");
        const double dtOut = o.interval > 0 ? o.interval : rec.dt;
        const double us = dtOut * 1e6;
        expect(dtOut > 0 && us <= 65535 && (!legacy || us >= 1), "SEG-Y sample interval must be positive and at most 65535 microseconds.");
        expect(!legacy || std::fabs(us - std::round(us)) < 1e-7,
               "Legacy SEG-Y requires whole-microsecond dt; select 0.5 or 1 ms output sampling.");
        const std::size_t nIn = rec.samples;
        expect(nIn > 0, "SEG-Y export requires nonempty traces.");
        const bool resample = dtOut != rec.dt;
        const double nOutReal = resample ? std::floor((nIn - 1) * rec.dt / dtOut + 1e-9) + 1 : static_cast<double>(nIn);
        expect(std::isfinite(nOutReal) && nOutReal >= 1 && nOutReal <= 65535, "SEG-Y export requires 1..65535 output samples per trace.");
        const auto nOut = static_cast<std::size_t>(nOutReal);
        expect(rec.traces.size() <= 100000, "Too many SEG-Y traces.");
        for (const auto &tr : rec.traces) {
            expect(tr.channel[component] != nullptr, "SEG-Y export requires equal trace lengths.");
            expect(std::isfinite(tr.start) && std::fabs(tr.start * 1000) <= 32767 &&
                       std::fabs(tr.start * 1000 - std::round(tr.start * 1000)) < 1e-7,
                   "SEG-Y export delay must be representable as whole milliseconds.");
            for (double v : tr.position) toMillimetres(v);
            for (double v : tr.source) toMillimetres(v);
            for (std::size_t t = 0; t < nIn; ++t) {
                const double v = tr.channel[component][t];
                expect(std::isfinite(v) && std::isfinite(v * o.gain) &&
                           (ieee64 || ibm || std::fabs(v * o.gain) <= std::numeric_limits<float>::max()),
                       "SEG-Y samples/multiplier overflow the selected precision.");
            }
        }
        // output sample t: the input at t (times the gain), or linear interpolation at t * dtOut
        const auto sampleAt = [&](const Trace &tr, std::size_t t) {
            const double *x = tr.channel[component];
            if (!resample) return x[t] * o.gain;
            const double u = std::clamp(t * dtOut / rec.dt, 0.0, static_cast<double>(nIn - 1));
            const auto i = static_cast<std::size_t>(u);
            return std::lerp(x[i], x[std::min(i + 1, nIn - 1)], u - i) * o.gain;
        };
        double peak = 0;
        std::size_t underflow = 0;
        for (const auto &tr : rec.traces)
            for (std::size_t t = 0; t < nOut; ++t) {
                const double v = sampleAt(tr, t);
                peak = std::max(peak, std::fabs(v));
                if (ibm) underflow += v != 0 && toIbm32(v) == 0;
                else if (!ieee64) underflow += v != 0 && static_cast<float>(v) == 0;
            }

        if (!path.parent_path().empty()) std::filesystem::create_directories(path.parent_path());
        partial = path;
        partial += ".partial";
        for (int k = 1; std::filesystem::exists(partial); ++k) {
            partial = path;
            partial += ".partial" + std::to_string(k);
        }
        std::ofstream out(partial, std::ios::binary);
        expect(static_cast<bool>(out), "Cannot create SEG-Y output.");

        Block text(3200, ' ');
        const auto card = [&](int row, const std::string &content) {
            const std::string line = "C" + std::string(row < 10 ? " " : "") + std::to_string(row) + " " + content;
            std::memcpy(text.bytes.data() + (row - 1) * 80, line.data(), std::min<std::size_t>(80, line.size()));
        };
        const std::string units = o.gain == 1 ? rec.units : "scaled(" + rec.units + ")";
        card(1, "SEISWAVE LAB - ELASTIC WAVE RECEIVER RECORDS");
        card(2, "COMPONENT=" + rec.components[component] + " UNITS=" + units);
        card(3, "EXACT DT (SECONDS)=" + exact(dtOut));
        card(4, std::string("SEG-Y REV ") + (legacy ? "1.0" : "2.0") + ", BIG ENDIAN, " + (ibm ? "IBM32" : ieee64 ? "IEEE64" : "IEEE32"));
        card(5, legacy ? "DT: BINARY BYTES 3217-3218; TRACE BYTES 117-118 (MICROSECONDS)"
                       : "EXACT DT: BINARY HEADER BYTES 3273-3280 (IEEE64 MICROSECONDS)");
        card(6, "COORDINATES/ELEVATIONS IN METRES; SCALARS=-1000; Z POSITIVE DOWN");
        card(7, "NO DISPLAY AGC OR TRACE NORMALIZATION; FIRST INPUT SAMPLE INCLUDED");
        card(8, "X IS INLINE, Y CROSSLINE; ONE VELOCITY COMPONENT PER FILE");
        card(9, "EXPORT_MULTIPLIER=" + exact(o.gain) + "; ORIGINAL_VALUE=STORED_VALUE/MULTIPLIER");
        card(10, "FFID=1; CHANNEL=1..N; CDP=1..N (ORDINAL, NOT A BINNED CMP GRID)");
        card(11, "SOURCE_DT_SECONDS=" + exact(rec.dt) + "; RESAMPLING=" + (resample ? "LINEAR" : "NONE"));
        card(12, "OUTPUT_PEAK=" + exact(peak) + "; UNDERFLOWED_SAMPLES=" + std::to_string(underflow));
        card(13, legacy ? "TRACE_ID=1 LIVE SEISMIC; COMPONENT IDENTIFIED ON C 2 / FILENAME"
                        : "TRACE_ID: 12=VERTICAL, 14=INLINE; COMPONENT IDENTIFIED ON C 2");
        card(40, "END TEXTUAL HEADER");
        if (ibm)
            for (auto &c : text.bytes) c = kCp037[c < 128 ? c : '?'];
        writeAll(out, text.bytes);

        const std::size_t n = rec.traces.size();
        const auto interval = static_cast<std::uint16_t>(std::clamp(std::llround(us), 1LL, 65535LL));
        Block bin(400);
        bin.put(12, std::min<std::size_t>(65535, n), 2); // data traces per ensemble
        bin.put(16, interval, 2);
        bin.put(18, interval, 2);
        bin.put(20, nOut, 2);
        bin.put(22, nOut, 2);
        bin.put(24, ibm ? 1 : ieee64 ? 6 : 5, 2); // sample format code
        bin.put(26, 1, 2);                         // ensemble fold
        bin.put(28, 1, 2);                         // sorting: as recorded
        bin.put(54, 1, 2);                         // metres
        if (!legacy) {
            bin.put(60, n, 4);
            bin.put(68, nOut, 4);
            bin.put(72, std::bit_cast<std::uint64_t>(us), 8);
            bin.put(80, std::bit_cast<std::uint64_t>(us), 8);
            bin.put(88, nOut, 4);
            bin.put(96, 0x01020304, 4); // byte-order marker
        }
        bin.bytes[300] = legacy ? 1 : 2; // revision
        bin.put(302, 1, 2);              // fixed-length traces
        if (!legacy) {
            bin.put(312, n, 8);
            bin.put(320, 3600, 8); // first trace header offset
        }
        writeAll(out, bin.bytes);

        const std::string &name = rec.components[component];
        const int traceId = legacy ? 1 : name == "Vz" ? 12 : name == "Vx" ? 14 : 1;
        const int unitCode = o.gain != 1 ? 0 : rec.units == "m/s" ? 6 : rec.units == "Pa" ? 1 : 0;
        const int width = ieee64 ? 8 : 4;
        for (std::size_t r = 0; r < n; ++r) {
            const Trace &tr = rec.traces[r];
            Block h(240);
            h.put(0, r + 1, 4);  // sequence in line
            h.put(4, r + 1, 4);  // sequence in file
            h.put(8, 1, 4);      // field record
            h.put(12, r + 1, 4); // channel
            h.put(16, 1, 4);     // energy source point
            h.put(20, r + 1, 4); // ensemble
            h.put(24, 1, 4);     // trace in ensemble
            h.put(28, traceId, 2);
            h.put(30, 1, 2), h.put(32, 1, 2), h.put(34, 1, 2);
            const double ox = tr.position[0] - tr.source[0], oy = tr.position[1] - tr.source[1];
            const double offset = std::copysign(std::hypot(ox, oy), ox != 0 ? ox : oy);
            expect(std::fabs(offset) <= std::numeric_limits<std::int32_t>::max(), "SEG-Y offset exceeds Int32 metres.");
            h.i32(36, static_cast<std::int32_t>(std::llround(offset)));
            h.i32(40, toMillimetres(-tr.position[2])); // receiver elevation
            h.i32(48, toMillimetres(tr.source[2]));    // source depth
            h.put(68, static_cast<std::uint16_t>(-1000), 2);
            h.put(70, static_cast<std::uint16_t>(-1000), 2);
            h.i32(72, toMillimetres(tr.source[0]));
            h.i32(76, toMillimetres(tr.source[1]));
            h.i32(80, toMillimetres(tr.position[0]));
            h.i32(84, toMillimetres(tr.position[1]));
            h.put(88, 1, 2); // coordinate units: length
            h.put(108, static_cast<std::uint16_t>(std::llround(tr.start * 1000)), 2);
            h.put(114, nOut, 2);
            h.put(116, interval, 2);
            h.i32(180, toMillimetres((tr.source[0] + tr.position[0]) * .5)); // midpoint
            h.i32(184, toMillimetres((tr.source[1] + tr.position[1]) * .5));
            h.put(202, unitCode, 2);
            writeAll(out, h.bytes);
            Block s(nOut * width);
            for (std::size_t t = 0; t < nOut; ++t) {
                const double v = sampleAt(tr, t);
                if (ibm) s.put(t * 4, toIbm32(v), 4);
                else if (ieee64) s.put(t * 8, std::bit_cast<std::uint64_t>(v), 8);
                else s.put(t * 4, std::bit_cast<std::uint32_t>(static_cast<float>(v)), 4);
            }
            writeAll(out, s.bytes);
        }
        out.close();
        expect(static_cast<bool>(out), "SEG-Y final flush failed.");
        std::filesystem::rename(partial, path);
    } catch (...) {
        if (!partial.empty()) {
            std::error_code ec;
            std::filesystem::remove(partial, ec);
        }
        throw;
    }
}

Imported readSegy(const std::filesystem::path &path) {
    std::ifstream in(path, std::ios::binary);
    expect(static_cast<bool>(in), "Cannot open SEG-Y input.");
    const auto size = std::filesystem::file_size(path);
    expect(size >= 3600, "SEG-Y input is shorter than its file headers.");
    const auto take = [&](std::size_t n) {
        Bytes b(n);
        expect(static_cast<bool>(in.read(reinterpret_cast<char *>(b.data()), static_cast<std::streamsize>(n))),
               "Truncated SEG-Y header or sample data.");
        return b;
    };
    const Bytes text = take(3200), binary = take(400);
    Fields big{binary, false};
    const auto marker = big.u(96, 4);
    expect(marker == 0 || marker == 0x01020304 || marker == 0x04030201,
           "Unsupported SEG-Y byte ordering (pair-swapped files are not supported).");
    bool little = marker == 0x04030201;
    if (!marker && !bytesPerSample(static_cast<int>(big.u(24, 2))) && bytesPerSample(static_cast<int>(Fields{binary, true}.u(24, 2))))
        little = true; // rev 0/1 file written little endian
    const Fields b{binary, little};
    const int format = static_cast<int>(b.u(24, 2)), width = bytesPerSample(format), revision = binary[300];
    expect(width > 0, "Unsupported SEG-Y sample format. Supported codes: 1,2,3,5,6,8.");
    expect(revision <= 2, "Unsupported SEG-Y revision.");
    expect(revision < 2 || b.u(306, 4) == 0,
           "SEG-Y additional trace headers are not supported; convert to standard 240-byte trace headers.");
    std::uint64_t offset = 3600;
    const int extended = revision ? b.s16(304) : 0;
    if (revision >= 2 && b.u(320, 8)) {
        offset = b.u(320, 8);
    } else {
        expect(extended >= 0 && extended <= 1024, "SEG-Y needs an explicit, bounded extended textual header count.");
        offset += static_cast<std::uint64_t>(extended) * 3200;
    }
    expect(offset >= 3600 && offset <= size, "SEG-Y first trace offset is outside the file.");
    in.seekg(static_cast<std::streamoff>(offset));
    const auto trailer = revision >= 2 ? b.s32(328) : 0;
    expect(trailer >= 0, "SEG-Y variable trailer counts are not supported.");
    expect(static_cast<std::uint64_t>(trailer) * 3200 <= size - offset, "Invalid SEG-Y data trailer size.");
    const auto end = size - static_cast<std::uint64_t>(trailer) * 3200;
    std::uint64_t samplesPerTrace = b.u(20, 2);
    if (revision >= 2 && b.u(68, 4)) samplesPerTrace = b.u(68, 4);
    double fileInterval = static_cast<double>(b.u(16, 2));
    if (revision >= 2 && b.f64(72) != 0) fileInterval = b.f64(72);
    const bool fixedLength = revision && b.u(302, 2) == 1;
    const double feet = b.u(54, 2) == 2 ? .3048 : 1;

    // textual header as ASCII (EBCDIC when it starts with an EBCDIC 'C')
    std::string card(text.begin(), text.end());
    if (text.front() == kCp037['C'])
        for (std::size_t i = 0; i < text.size(); ++i) {
            const auto *hit = std::find(std::begin(kCp037), std::end(kCp037), text[i]);
            card[i] = hit == std::end(kCp037) ? '?' : static_cast<char>(hit - std::begin(kCp037));
        }
    const bool ours = card.find("SEISWAVE LAB") != std::string::npos;
    const auto keyOnLine2 = [&](const char *key) { // value after `key` on card 2, up to a space
        const std::string line = card.substr(80, 80);
        const auto at = line.find(key);
        if (at == std::string::npos) return std::string();
        const auto from = at + std::strlen(key);
        return line.substr(from, line.find(' ', from) - from);
    };
    Imported result;
    if (ours && !keyOnLine2("UNITS=").empty()) result.units = keyOnLine2("UNITS=");
    std::size_t decodedBytes = 0;
    int traceId = -1, unitCode = -1;
    while (offset < end) {
        expect(result.traces.size() < 4096, "SEG-Y import exceeds 4096 trace positions.");
        expect(end - offset >= 240, "Incomplete SEG-Y trace header.");
        const Bytes hb = take(240);
        offset += 240;
        const Fields h{hb, little};
        const std::uint64_t count = fixedLength ? samplesPerTrace : (h.u(114, 2) ? h.u(114, 2) : samplesPerTrace);
        expect(count > 0 && count <= 1000000 && count <= ((256ULL << 20) - decodedBytes) / sizeof(double),
               "SEG-Y sample count exceeds the import memory budget (256 MiB).");
        double interval = fixedLength && fileInterval > 0 ? fileInterval : static_cast<double>(h.u(116, 2));
        if (interval == 0) interval = fileInterval;
        expect(std::isfinite(interval) && interval >= 1e-6 && interval <= 1e9,
               "SEG-Y sample interval is missing, invalid or outside 1 ps..1000 s.");
        if (result.traces.empty()) result.dt = interval * 1e-6;
        else
            expect(std::fabs(result.dt - interval * 1e-6) <= std::max(1e-12, result.dt * 1e-9),
                   "SEG-Y traces have different sample intervals; resample before import.");
        expect(count * width <= end - offset, "Truncated SEG-Y trace samples.");
        const Bytes sb = take(static_cast<std::size_t>(count) * width);
        offset += count * width;
        decodedBytes += count * sizeof(double);
        const Fields s{sb, little};
        ImportedTrace tr;
        const double xy = headerScale(h.s16(70)), elevation = headerScale(h.s16(68));
        expect(h.u(88, 2) <= 1, "SEG-Y angular coordinates are not supported in this Cartesian record viewer.");
        tr.position = {h.s32(80) * xy * feet, h.s32(84) * xy * feet, -static_cast<double>(h.s32(40)) * elevation * feet};
        tr.source = {h.s32(72) * xy * feet, h.s32(76) * xy * feet, (h.s32(48) - static_cast<double>(h.s32(44))) * elevation * feet};
        tr.start = h.s16(108) * .001 * (revision ? headerScale(h.s16(214)) : 1);
        const int weighting = h.s16(168);
        expect(weighting >= -1022 && weighting <= 1022, "SEG-Y trace weighting is outside the supported finite range.");
        tr.samples.resize(count);
        for (std::size_t t = 0; t < count; ++t) {
            const std::size_t at = t * width;
            double v;
            switch (format) {
            case 5: v = std::bit_cast<float>(static_cast<std::uint32_t>(s.u(at, 4))); break;
            case 6: v = s.f64(at); break;
            case 2: v = s.s32(at); break;
            case 3: v = s.s16(at); break;
            case 8: v = std::bit_cast<std::int8_t>(sb[at]); break;
            default: v = fromIbm32(static_cast<std::uint32_t>(s.u(at, 4))); break;
            }
            v = std::ldexp(v, -weighting);
            expect(std::isfinite(v), "SEG-Y contains nonfinite samples.");
            tr.samples[t] = v;
        }
        const int id = static_cast<int>(h.u(28, 2));
        traceId = traceId < 0 ? id : traceId != id ? 0 : traceId;
        const int unit = revision ? h.s16(202) : 0;
        unitCode = unitCode < 0 ? unit : unitCode != unit ? 1000 : unitCode;
        result.traces.push_back(std::move(tr));
    }
    expect(!result.traces.empty(), "SEG-Y contains no data traces.");
    result.component = traceId == 12 ? "Vz" : traceId == 14 ? "Vx" : "Amplitude";
    if (ours && !keyOnLine2("COMPONENT=").empty()) result.component = keyOnLine2("COMPONENT=");
    static const char *const kUnits[] = {"raw", "Pa", "V", "mV", "A", "m", "m/s", "m/s2", "N", "W"};
    if (unitCode > 0 && unitCode < 10) result.units = kUnits[unitCode];
    if (unitCode == 1000) result.units = "mixed";
    result.description = "SEG-Y rev " + std::to_string(revision) + " | format " + std::to_string(format) +
                         (little ? " | little endian" : " | big endian");
    return result;
}

} // namespace swl::records

// ------------------------------------------------------------------------------------ C ABI
struct swl_segy_records : swl::records::Imported {};

namespace {
template <class F> swl_status recordsGuard(F &&f) {
    std::string &err = swl::lastErrorRef();
    try {
        err.clear();
        f();
        return SWL_OK;
    } catch (const std::bad_alloc &) {
        err = "host allocation failed";
        return SWL_ERR_MEMORY;
    } catch (const std::exception &e) {
        err = e.what();
        return SWL_ERR_INVALID;
    }
}
void copyText(char *dst, std::size_t cap, const std::string &s) {
    const std::size_t n = std::min(cap - 1, s.size());
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
}
} // namespace

extern "C" {
void swl_segy_options_default(swl_segy_options *o) {
    if (o) *o = swl_segy_options{SWL_SEGY_IEEE32, 1.0, 0.0};
}
swl_status swl_write_segy(const swl_record_view *v, int32_t component, const char *path, const swl_segy_options *o) {
    return recordsGuard([&] {
        if (!v || !path || !o) throw std::runtime_error("records, path and options are required");
        if (v->n_traces < 0 || v->n_components < 1 || v->n_components > 3 || v->n_samples < 0 || (v->n_traces && !v->traces))
            throw std::runtime_error("invalid record view");
        swl::records::RecordSet rec;
        rec.dt = v->dt, rec.samples = std::size_t(v->n_samples);
        if (v->units) rec.units = v->units;
        for (int c = 0; c < v->n_components; ++c) rec.components.emplace_back(v->components[c] ? v->components[c] : "");
        for (int r = 0; r < v->n_traces; ++r) {
            const swl_trace_view &t = v->traces[r];
            swl::records::Trace tr;
            std::copy(t.position, t.position + 3, tr.position.begin());
            std::copy(t.source, t.source + 3, tr.source.begin());
            tr.start = t.start_time;
            for (int c = 0; c < v->n_components; ++c) tr.channel[c] = t.channels[c];
            rec.traces.push_back(tr);
        }
        swl::records::writeSegy(rec, component, path, {o->profile, o->sample_gain, o->sample_interval_s});
    });
}
swl_status swl_read_segy(const char *path, swl_segy_records **out) {
    return recordsGuard([&] {
        if (!path || !out) throw std::runtime_error("path and out are required");
        *out = nullptr;
        auto r = std::make_unique<swl_segy_records>();
        static_cast<swl::records::Imported &>(*r) = swl::records::readSegy(path);
        *out = r.release();
    });
}
void swl_segy_records_free(swl_segy_records *r) { delete r; }
swl_status swl_segy_records_info(const swl_segy_records *r, swl_segy_info *o) {
    return recordsGuard([&] {
        if (!r || !o) throw std::runtime_error("records and out are required");
        *o = swl_segy_info{};
        o->n_traces = int32_t(r->traces.size());
        for (const auto &t : r->traces) o->max_samples = std::max<int64_t>(o->max_samples, int64_t(t.samples.size()));
        o->dt = r->dt;
        copyText(o->component, sizeof o->component, r->component);
        copyText(o->units, sizeof o->units, r->units);
        copyText(o->description, sizeof o->description, r->description);
    });
}
swl_status swl_segy_records_trace(const swl_segy_records *r, int32_t index, double position[3], double source[3],
                                  double *start_time, double *samples, int64_t capacity, int64_t *n_samples) {
    return recordsGuard([&] {
        if (!r) throw std::runtime_error("records are required");
        if (index < 0 || std::size_t(index) >= r->traces.size()) throw std::runtime_error("trace index out of range");
        const auto &t = r->traces[index];
        if (position) std::copy(t.position.begin(), t.position.end(), position);
        if (source) std::copy(t.source.begin(), t.source.end(), source);
        if (start_time) *start_time = t.start;
        if (n_samples) *n_samples = int64_t(t.samples.size());
        if (samples) std::copy_n(t.samples.begin(), std::min<std::size_t>(t.samples.size(), std::size_t(std::max<int64_t>(0, capacity))), samples);
    });
}
} // extern "C"

// GSLS (generalized standard linear solid) fit and the PCHIP terrain profile.
#include "model.hpp"
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <stdexcept>

namespace swl::host {
namespace {
constexpr double pi = 3.14159265358979323846;
void require(bool ok, const char *message) {
    if (!ok) throw std::runtime_error(message);
}

// Relaxation strengths for one quality factor: exhaustive active-set non-negative least squares
// of the 1/Q misfit over 81 log-spaced frequencies (src/common/Gsls.cpp:11-33).
std::array<double, 3> strengths(double q, const GslsMaterial &m, const GslsSettings &s) {
    constexpr int samples = 81;
    double design[samples][3]{};
    const double target = 1 / q;
    for (int i = 0; i < samples; ++i) {
        const double w = 2 * pi * s.minFrequency * std::pow(s.maxFrequency / s.minFrequency, double(i) / (samples - 1));
        for (int l = 0; l < m.mechanisms; ++l) {
            const double x = w / m.rates[l];
            design[i][l] = (x - target * x * x) / (1 + x * x);
        }
    }
    std::array<double, 3> best{};
    double bestCost = std::numeric_limits<double>::infinity();
    for (int mask = 1; mask < (1 << m.mechanisms); ++mask) {
        int ids[3]{}, n = 0;
        for (int l = 0; l < m.mechanisms; ++l)
            if (mask & (1 << l)) ids[n++] = l;
        // normal equations [A | b] of the active columns
        double a[3][4]{};
        for (int i = 0; i < n; ++i)
            for (int row = 0; row < samples; ++row) {
                a[i][n] += design[row][ids[i]] * target;
                for (int j = 0; j < n; ++j) a[i][j] += design[row][ids[i]] * design[row][ids[j]];
            }
        // Gauss-Jordan elimination with partial pivoting
        bool valid = true;
        for (int k = 0; k < n; ++k) {
            int pivot = k;
            for (int i = k + 1; i < n; ++i)
                if (std::abs(a[i][k]) > std::abs(a[pivot][k])) pivot = i;
            if (std::abs(a[pivot][k]) < 1e-20) {
                valid = false;
                break;
            }
            for (int j = 0; j <= n; ++j) std::swap(a[k][j], a[pivot][j]);
            const double d = a[k][k];
            for (int j = k; j <= n; ++j) a[k][j] /= d;
            for (int i = 0; i < n; ++i)
                if (i != k) {
                    const double f = a[i][k];
                    for (int j = k; j <= n; ++j) a[i][j] -= f * a[k][j];
                }
        }
        std::array<double, 3> candidate{};
        for (int i = 0; i < n && valid; ++i) {
            valid = std::isfinite(a[i][n]) && a[i][n] >= 0;
            candidate[ids[i]] = a[i][n];
        }
        if (!valid) continue;
        double cost = 0;
        for (int row = 0; row < samples; ++row) {
            double residual = -target;
            for (int l = 0; l < m.mechanisms; ++l) residual += design[row][l] * candidate[l];
            cost += residual * residual;
        }
        if (cost < bestCost) bestCost = cost, best = candidate;
    }
    require(std::isfinite(bestCost), "No passive GSLS fit for this Q/frequency band.");
    return best;
}
std::complex<double> modulus(const GslsMaterial &m, bool shear, std::complex<double> s) {
    std::complex<double> c = shear ? m.sRelaxed : m.pRelaxed;
    for (int l = 0; l < m.mechanisms; ++l) c += (shear ? m.deltaS[l] : m.deltaP[l]) * s / (s + m.rates[l]);
    return c;
}
} // namespace

// src/common/Gsls.cpp:28-33
void validateGsls(const GslsSettings &s) {
    require(s.mechanisms >= 1 && s.mechanisms <= 3, "GSLS mechanism count must be 1..3.");
    require(std::isfinite(s.minFrequency) && std::isfinite(s.maxFrequency) && std::isfinite(s.referenceFrequency) &&
                s.minFrequency > 0 && s.maxFrequency > s.minFrequency && s.maxFrequency <= 1e6 && s.minFrequency >= .01 &&
                s.referenceFrequency >= s.minFrequency && s.referenceFrequency <= s.maxFrequency,
            "GSLS requires 0.01 <= fmin < fmax <= 1e6 Hz and fref within the band.");
    for (double q : {s.qp, s.qs})
        require(std::isfinite(q) && q >= 5 && q <= 1e9,
                "Qp and Qs must be finite and in 5..1e9; disable attenuation for the elastic limit.");
}

// src/common/Gsls.cpp:34-35
double gslsQuality(const GslsMaterial &m, bool shear, double f) {
    const auto c = modulus(m, shear, {0, 2 * pi * f});
    return c.real() / std::abs(c.imag());
}

// src/common/Gsls.cpp:38-54 -- log-spaced rates, strengths, moduli scaled so the phase
// velocity at the reference frequency equals the given velocity, passivity checks.
GslsMaterial fitGsls(double vp, double vs, double rho, double qp, double qs, const GslsSettings &settings) {
    validateGsls(settings);
    require(std::isfinite(vp) && std::isfinite(vs) && std::isfinite(rho) && rho > 0 && vs > 0 && vp * vp > 4 * vs * vs / 3,
            "Invalid GSLS reference velocities/density.");
    for (double q : {qp, qs}) require(std::isfinite(q) && q >= 5 && q <= 1e9, "Layer Qp/Qs must be in 5..1e9.");
    GslsMaterial m;
    m.mechanisms = settings.mechanisms;
    for (int l = 0; l < m.mechanisms; ++l)
        m.rates[l] = 2 * pi *
                     (m.mechanisms == 1 ? std::sqrt(settings.minFrequency * settings.maxFrequency)
                                        : settings.minFrequency *
                                              std::pow(settings.maxFrequency / settings.minFrequency, double(l) / (m.mechanisms - 1)));
    const auto p = strengths(qp, m, settings), s = strengths(qs, m, settings);
    const std::complex<double> w{0, 2 * pi * settings.referenceFrequency};
    const auto scale = [&](const std::array<double, 3> &weights, double velocity) {
        std::complex<double> shape = 1.;
        for (int l = 0; l < m.mechanisms; ++l) shape += weights[l] * w / (w + m.rates[l]);
        const double inv = std::real(1. / std::sqrt(shape));
        return rho * velocity * velocity * inv * inv;
    };
    m.pRelaxed = scale(p, vp);
    m.sRelaxed = scale(s, vs);
    m.pUnrelaxed = m.pRelaxed;
    m.sUnrelaxed = m.sRelaxed;
    require(m.pRelaxed > 4 * m.sRelaxed / 3, "Qp/Qs produce nonpositive relaxed bulk modulus.");
    for (int l = 0; l < m.mechanisms; ++l) {
        m.deltaP[l] = m.pRelaxed * p[l];
        m.deltaS[l] = m.sRelaxed * s[l];
        require(m.deltaP[l] + 1e-12 * m.pRelaxed >= 4 * m.deltaS[l] / 3,
                "Qp/Qs violate passive bulk relaxation (Qp cannot be arbitrarily large relative to Qs).");
        m.pUnrelaxed += m.deltaP[l];
        m.sUnrelaxed += m.deltaS[l];
    }
    require(std::isfinite(m.pUnrelaxed) && std::isfinite(m.sUnrelaxed), "GSLS moduli overflow.");
    for (int i = 0; i <= 160; ++i) {
        const double f = settings.minFrequency * std::pow(settings.maxFrequency / settings.minFrequency, i / 160.);
        m.maxRelativeQError = std::max({m.maxRelativeQError, std::abs(gslsQuality(m, false, f) / qp - 1),
                                        std::abs(gslsQuality(m, true, f) / qs - 1)});
    }
    return m;
}

// src/two_d/SurfaceProfile.cpp:8-49 -- monotone cubic Hermite (PCHIP) slopes with the
// three-point end formula.
SurfaceProfile::SurfaceProfile(const std::vector<std::array<double, 2>> &points) : points_(points) {
    require(points.size() >= 2 && points.size() <= 1000000, "Surface profile requires 2..1000000 samples.");
    std::vector<double> h(points.size() - 1), d(h.size());
    for (std::size_t i = 0; i < points.size(); ++i) {
        require(std::isfinite(points[i][0]) && std::isfinite(points[i][1]) && (!i || points[i][0] > points[i - 1][0]),
                "Surface samples must be finite with strictly increasing x.");
        if (i) {
            h[i - 1] = points[i][0] - points[i - 1][0];
            d[i - 1] = (points[i][1] - points[i - 1][1]) / h[i - 1];
            require(std::isfinite(h[i - 1]) && std::isfinite(d[i - 1]), "Surface sample differences overflow.");
        }
    }
    slopes_.assign(points.size(), 0);
    slopes_.front() = d.front();
    slopes_.back() = d.back();
    if (points.size() == 2) return;
    const auto endpoint = [](double h0, double h1, double d0, double d1) {
        const double m = ((2 * h0 + h1) * d0 - h0 * d1) / (h0 + h1);
        if (m * d0 <= 0) return 0.0;
        if (d0 * d1 < 0 && std::abs(m) > 3 * std::abs(d0)) return 3 * d0;
        return m;
    };
    const std::size_t n = h.size();
    slopes_.front() = endpoint(h[0], h[1], d[0], d[1]);
    slopes_.back() = endpoint(h[n - 1], h[n - 2], d[n - 1], d[n - 2]);
    for (std::size_t i = 1; i + 1 < points.size(); ++i) {
        if (d[i - 1] * d[i] <= 0) slopes_[i] = 0;
        else {
            const double a = 2 * h[i] + h[i - 1], b = h[i] + 2 * h[i - 1];
            slopes_[i] = (a + b) / (a / d[i - 1] + b / d[i]);
        }
    }
    for (double s : slopes_) require(std::isfinite(s), "Surface interpolation coefficients overflow.");
}

// src/two_d/SurfaceProfile.cpp:50-64 -- linear continuation outside the samples.
std::array<double, 2> SurfaceProfile::sample(double x) const {
    if (x <= points_.front()[0]) return {points_.front()[1] + (x - points_.front()[0]) * slopes_.front(), slopes_.front()};
    if (x >= points_.back()[0]) return {points_.back()[1] + (x - points_.back()[0]) * slopes_.back(), slopes_.back()};
    const auto upper =
        std::upper_bound(points_.begin(), points_.end(), x, [](double value, const auto &p) { return value < p[0]; });
    const auto i = static_cast<std::size_t>(upper - points_.begin() - 1);
    const double h = points_[i + 1][0] - points_[i][0], t = (x - points_[i][0]) / h;
    const double a = points_[i][1], b = points_[i + 1][1], m = slopes_[i], n = slopes_[i + 1];
    return {(2 * t * t * t - 3 * t * t + 1) * a + (t * t * t - 2 * t * t + t) * h * m + (-2 * t * t * t + 3 * t * t) * b +
                (t * t * t - t * t) * h * n,
            (6 * t * t - 6 * t) * (a - b) / h + (3 * t * t - 4 * t + 1) * m + (3 * t * t - 2 * t) * n};
}

// include/Seis3D/SurfaceGrid3D.hpp:44-51 -- bilinear DEM with edge-cell extension.
double SurfaceGrid3D::elevation(double x, double y) const {
    const double u = x / spacing, v = y / spacing;
    const int i = static_cast<int>(std::floor(std::clamp(u, 0.0, static_cast<double>(nx - 2))));
    const int j = static_cast<int>(std::floor(std::clamp(v, 0.0, static_cast<double>(ny - 2))));
    const double a = u - i, b = v - j;
    const auto at = [&](int ix, int iy) { return elevations[static_cast<std::size_t>(iy) * nx + ix]; };
    return (1 - b) * ((1 - a) * at(i, j) + a * at(i + 1, j)) + b * ((1 - a) * at(i, j + 1) + a * at(i + 1, j + 1));
}

} // namespace swl::host

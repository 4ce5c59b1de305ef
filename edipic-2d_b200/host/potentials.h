// Potential of one metal electrode as a function of the time step: UPDATE_WALL_POTENTIALS with its three parts,
// Harmonic_Oscillation, Custom_Waveform and Amplitude_Profile (pic2d_WallPotentials.f90:1-165), and the readers of
// the two optional files that set them up, init_bo_NN_waveform.dat (PREPARE_WAVEFORMS, pic2d_Setup.f90:150-269) and
// init_bo_NN_amplitude_profile.dat (PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE, pic2d_Setup.f90:273-412).
//
// The reference keeps the waveform values and amplitude factors, and the interpolation weight, in single precision
// (REAL); the same rounding is kept here so that the potential matches for the same files. Header-only: the deck
// reader (host/deck.cpp) and the device context (csrc/edp_api.cu) share it.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

struct EdpPotentialProfile {
    double phi_const = 0.0, phi_var = 0.0;   // normalised by F_scale
    double omega = 0.0;                      // rad per time step
    double phase = 0.0, phase_adjusted = 0.0;
    std::vector<int32_t> wf_t;               // Custom_Waveform: time steps of the points (use_waveform if non-empty)
    std::vector<float> wf_phi;               //   potentials of the points, normalised
    std::vector<int32_t> ap_t;               // Amplitude_Profile: time steps (use_amplitude_profile if non-empty)
    std::vector<float> ap_factor;            //   amplitude factors

    static constexpr double kPi = 3.141592653589793;

    // Harmonic_Oscillation (:58-93): with an amplitude profile, the phase is re-anchored at the start of every
    // profile period so that each pulse starts with the same phase
    double harmonic(int32_t t)
    {
        if (!ap_t.empty()) {
            const int32_t period = ap_t.back();
            if (t == (t / period) * period) {
                const int32_t n_periods = (int32_t)((omega * (double)t) / (2.0 * kPi));
                phase_adjusted = (double)n_periods * 2.0 * kPi + phase - omega * (double)t;
            }
            return phi_var * std::sin(omega * (double)t + phase_adjusted);
        }
        return phi_var * std::sin(omega * (double)t + phase);
    }

    // linear interpolation between the points of a periodic table, with the reference's single-precision weight:
    // v(i) * ai is a REAL product, v(i+1) * (1 - ai) a REAL(8) one
    static bool interpolate(const std::vector<int32_t>& tt, const std::vector<float>& v, int32_t t, double* out)
    {
        const int32_t period = tt.back();
        const int32_t my = t - (t / period) * period;
        for (size_t i = 0; i + 1 < tt.size(); ++i) {
            if (my >= tt[i] && my <= tt[i + 1]) {
                const float ai = (float)((double)(tt[i + 1] - my) / (double)(tt[i + 1] - tt[i]));
                const float first = v[i] * ai;
                const double second = (double)v[i + 1] * (1.0 - (double)ai);
                *out = (double)first + second;
                return true;
            }
        }
        return false;
    }

    // Custom_Waveform (:95-128): 0 without a waveform
    double waveform(int32_t t) const
    {
        double r = 0.0;
        if (!wf_t.empty()) interpolate(wf_t, wf_phi, t, &r);
        return r;
    }

    // Amplitude_Profile (:132-165): 1 without a profile
    double amplitude(int32_t t) const
    {
        double r = 1.0;
        if (!ap_t.empty() && !interpolate(ap_t, ap_factor, t, &r)) r = 1.0;
        return r;
    }

    // UPDATE_WALL_POTENTIALS (:15-27) for this object at time step t; call it for consecutive t (the phase of a
    // pulsed oscillation is re-anchored as the steps pass period starts)
    double value(int32_t t) { return phi_const + (harmonic(t) + waveform(t)) * amplitude(t); }

    // ADJUST_HARMONIC_OSCILLATIONS_PHASE (:180-206): the phase of a run continued at step start_t
    void adjust_phase(int32_t start_t)
    {
        phase_adjusted = phase;
        if (start_t == 0 || ap_t.empty()) return;
        const int32_t period = ap_t.back();
        const int32_t my = (start_t / period) * period;
        const int32_t n_periods = (int32_t)((omega * (double)my) / (2.0 * kPi));
        phase_adjusted = (double)n_periods * 2.0 * kPi + phase - omega * (double)my;
    }
};

namespace edp_potentials_detail {

// the (x, y) pairs a list-directed READ (11, *) x, y takes from successive lines, from line `skip` on, until the
// first line that does not start with two numbers
inline std::vector<std::pair<std::string, std::string>> pairs(const std::vector<std::string>& lines, size_t skip)
{
    std::vector<std::pair<std::string, std::string>> out;
    for (size_t k = skip; k < lines.size(); ++k) {
        std::istringstream is(lines[k]);
        std::string a, b;
        if (!(is >> a)) continue;   // a blank record: list-directed input goes on to the next one
        if (!(is >> b)) break;
        char* e1 = nullptr;
        char* e2 = nullptr;
        std::string a2 = a, b2 = b;
        for (char& ch : a2) if (ch == 'd' || ch == 'D') ch = 'e';
        for (char& ch : b2) if (ch == 'd' || ch == 'D') ch = 'e';
        std::strtod(a2.c_str(), &e1);
        std::strtod(b2.c_str(), &e2);
        if (!e1 || *e1 || !e2 || *e2) break;
        out.emplace_back(a2, b2);
    }
    return out;
}

inline bool read_lines(const std::string& path, std::vector<std::string>* lines)
{
    std::ifstream f(path);
    if (!f) return false;
    std::string s;
    while (std::getline(f, s)) {
        if (!s.empty() && s.back() == '\r') s.pop_back();
        lines->push_back(s);
    }
    return true;
}

inline double first_number(const std::string& line, bool* ok)
{
    std::istringstream is(line);
    std::string a;
    *ok = false;
    if (!(is >> a)) return 0.0;
    for (char& ch : a) if (ch == 'd' || ch == 'D') ch = 'e';
    char* e = nullptr;
    double v = std::strtod(a.c_str(), &e);
    *ok = e && *e == 0;
    return v;
}

}  // namespace edp_potentials_detail

// PREPARE_WAVEFORMS (pic2d_Setup.f90:150-269) for one metal object: fills wf_t / wf_phi when the file exists and
// passes the reference's checks, else leaves them empty (the waveform is off, as the reference only warns)
inline void edp_read_waveform(const std::string& path, double delta_t_s, double f_scale_v, EdpPotentialProfile* p)
{
    using namespace edp_potentials_detail;
    p->wf_t.clear();
    p->wf_phi.clear();
    std::vector<std::string> L;
    if (!read_lines(path, &L) || L.size() < 4) return;
    const auto pts = pairs(L, 4);   // amplitude, frequency and two comment lines come first
    const size_t n = pts.size();
    if (n <= 1) return;
    bool ok1 = false, ok2 = false;
    const double phi_v = first_number(L[0], &ok1);
    const double nu_hz = first_number(L[1], &ok2);
    if (!ok1 || !ok2 || phi_v == 0.0) return;
    const int32_t period = (int32_t)(1.0 / (nu_hz * delta_t_s));   // integer number of time steps (truncated)
    if (period < (int32_t)(n - 1)) return;
    std::vector<int32_t> t(n);
    std::vector<float> v(n);
    for (size_t i = 0; i < n; ++i) {
        const float rd = std::strtof(pts[i].first.c_str(), nullptr);     // REAL rdummy
        const float ph = std::strtof(pts[i].second.c_str(), nullptr);    // REAL wf_phi(i)
        t[i] = (int32_t)(rd * (float)period);                             // REAL * INTEGER, truncated
        v[i] = (float)((phi_v / f_scale_v) * (double)ph);
    }
    t[0] = 0;
    t[n - 1] = period;
    for (size_t i = 1; i + 1 < n; ++i) t[i] = t[i] > t[i - 1] + 1 ? t[i] : t[i - 1] + 1;
    if (!(t[n - 1] > t[n - 2])) return;
    p->wf_t = t;
    p->wf_phi = v;
}

// PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE (pic2d_Setup.f90:273-412) for one metal object, after its waveform
inline void edp_read_amplitude_profile(const std::string& path, double delta_t_s, EdpPotentialProfile* p)
{
    using namespace edp_potentials_detail;
    p->ap_t.clear();
    p->ap_factor.clear();
    std::vector<std::string> L;
    if (!read_lines(path, &L) || L.empty()) return;
    const auto pts = pairs(L, 1);   // one comment line
    const size_t n = pts.size();
    if (n <= 1) return;
    std::vector<int32_t> t(n);
    std::vector<float> a(n);
    for (size_t i = 0; i < n; ++i) {
        const float rd = std::strtof(pts[i].first.c_str(), nullptr);
        a[i] = std::strtof(pts[i].second.c_str(), nullptr);
        t[i] = (int32_t)((double)rd * 1.0e-9 / delta_t_s);
    }
    t[0] = 0;
    for (size_t i = 1; i + 1 < n; ++i) t[i] = t[i] > t[i - 1] + 1 ? t[i] : t[i - 1] + 1;
    if (!p->wf_t.empty()) {
        // ends of the non-zero intervals moved to whole waveform periods
        const int32_t wp = p->wf_t.back();
        for (size_t i = 0; i + 1 < n; ++i) {
            if (a[i] == 0.0f && a[i + 1] != 0.0f) {
                const int32_t d = t[i + 1] - t[i];
                t[i] = wp * (t[i] / wp);
                t[i + 1] = t[i] + d;
            }
        }
        for (size_t i = 1; i < n; ++i) {
            if (a[i - 1] != 0.0f && a[i] == 0.0f) {
                const int32_t d = t[i] - t[i - 1];
                t[i] = wp * (t[i] / wp);
                t[i - 1] = t[i] - d;
            }
        }
        t[n - 1] = wp * (t[n - 1] / wp);
    }
    for (size_t i = 0; i + 1 < n; ++i)
        if (!(t[i + 1] > t[i])) return;   // inconsistent: the profile is off
    p->ap_t = t;
    p->ap_factor = a;
}

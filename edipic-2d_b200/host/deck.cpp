// Deck reader: the host side of INITIATE_PARAMETERS (pic2d_CurProblemValues.f90:59-1255) and of the collision
// set-up (pic2d_enCollisionsGeneralProc.f90:5-325, pic2d_inCollisionsGeneralProc.f90:3-90), reading the same
// fixed-column init_*.dat files with the same field widths, and producing edp_params / edp_tables.
//
// Supported deck subset: one cluster covering the domain (any block count), boundary objects that are metal
// walls (type 1) or periodic pipes (type 2) on the four sides, metal rectangular inner objects, uniform external
// B and Ez, one neutral species with e-n processes of types 10/11/20/30 and resonant charge exchange.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/edipic_gpu.h"
#include "potentials.h"

namespace {

const double E_CL = 1.602189e-19, M_E_KG = 9.109534e-31, TRUE_EPS0 = 8.854188e-12, AMU_KG = 1.660565e-27,
             KB_JK = 1.38064852e-23, PI = 3.141592653589793;

struct Lines {
    std::vector<std::string> v;
    size_t pos = 0;
    bool ok = false;
    explicit Lines(const std::string& path)
    {
        std::ifstream f(path);
        if (!f) return;
        std::string s;
        while (std::getline(f, s)) {
            if (!s.empty() && s.back() == '\r') s.pop_back();
            v.push_back(s);
        }
        ok = true;
    }
    bool next(std::string& s)
    {
        if (pos >= v.size()) return false;
        s = v[pos++];
        return true;
    }
};

// Fortran fixed-width field: columns [skip, skip+width) of the line, blanks ignored
std::string field(const std::string& line, size_t skip, size_t width)
{
    if (line.size() <= skip) return "";
    std::string f = line.substr(skip, width);
    std::string out;
    for (char ch : f)
        if (ch != ' ' && ch != '\t') out.push_back(ch);
    return out;
}
bool fint(const std::string& line, size_t skip, size_t width, long long* v)
{
    std::string f = field(line, skip, width);
    if (f.empty()) {
        *v = 0;
        return true;
    }
    char* e = nullptr;
    *v = strtoll(f.c_str(), &e, 10);
    return e && *e == 0;
}
bool freal(const std::string& line, size_t skip, size_t width, double* v)
{
    std::string f = field(line, skip, width);
    if (f.empty()) {
        *v = 0.0;
        return true;
    }
    for (char& ch : f)
        if (ch == 'd' || ch == 'D') ch = 'e';
    char* e = nullptr;
    *v = strtod(f.c_str(), &e);
    return e && *e == 0;
}

struct CrossSection {
    int type = 0;
    int activated = 0;
    int ion_species = 0;
    std::vector<double> e, s;
};

double en_frequency(const CrossSection& cs, double E, double n_m3, int nsub, double dt)
{
    // frequency_of_en_collision, pic2d_enCollisionsSpecificProc.f90:4-57
    const size_t N = cs.e.size();
    double f;
    if (E >= cs.e[N - 1]) f = cs.s[N - 1] * std::sqrt(2.0 * E * E_CL / M_E_KG);
    else if (E < cs.e[0]) f = (cs.type < 20) ? cs.s[0] * std::sqrt(2.0 * E * E_CL / M_E_KG) : 0.0;
    else {
        size_t j = 0;
        while (j + 1 < N && !(E >= cs.e[j] && E < cs.e[j + 1])) ++j;
        if (j > N - 2) j = N - 2;
        double fj = cs.s[j] * std::sqrt(2.0 * cs.e[j] * E_CL / M_E_KG);
        double fj1 = cs.s[j + 1] * std::sqrt(2.0 * cs.e[j + 1] * E_CL / M_E_KG);
        f = fj + (fj1 - fj) * (E - cs.e[j]) / (cs.e[j + 1] - cs.e[j]);
    }
    return f * n_m3 * nsub * dt;
}

}  // namespace

struct edp_deck {
    edp_params p;
    edp_tables t;
    std::vector<double> prob, energy, maxwell;
    double init_te = 0, init_ne = 0, init_ti[EDP_MAX_ION_SPECIES] = {0}, t_e = 0, n_plasma = 0;
    int32_t n_max_vel = 0;
    int64_t max_t_cntr = 0;
    // ion-induced electron emission of the four walls per ion species: yield, E_min [eV], E_max [eV], T [eV]
    // per object: the walls 0 below, 1 above, 2 left, 3 right, then inner object n at 4 + n
    double ii_ee[EDP_N_HIT_COUNTERS][EDP_MAX_ION_SPECIES][4] = {};
    int32_t ion_model[EDP_N_HIT_COUNTERS] = {};   // ion-material interaction model of the object's material
    edp_see_params see[EDP_N_HIT_COUNTERS] = {};  // electron-induced emission of the object's material
    // constant electron emission of each metal wall and inner object: N per step, model, T_n, T_p, W_beam [eV]
    double inject[EDP_N_HIT_COUNTERS][5] = {};
    // potentials of the metal objects over time (walls 0 below, 1 above, 2 left, 3 right; inner objects 4 + n)
    EdpPotentialProfile pot[4 + EDP_MAX_INNER];
};

namespace {

int read_deck(const std::string& dir, edp_deck* d)
{
    edp_params& p = d->p;
    edp_tables& t = d->t;
    memset(&p, 0, sizeof(p));
    memset(&t, 0, sizeof(t));
    p.abi_version = EDP_ABI_VERSION;
    std::string L;
    // ---- init_configuration.dat (pic2d_CurProblemValues.f90:157-330)
    // SET_PHYSICAL_CONSTANTS (pic2d_CurProblemValues.f90:3-55): eps_0 from init_physconstants.dat when it holds a
    // positive value on its second line, else the true value
    double EPS0 = TRUE_EPS0;
    {
        Lines pc(dir + "/init_physconstants.dat");
        std::string l1, l2;
        if (pc.ok && pc.next(l1) && pc.next(l2)) {
            bool ok = false;
            const double v = edp_potentials_detail::first_number(l2, &ok);   // READ (9, *) temp
            if (ok && v > 0.0) EPS0 = v;
        }
    }
    Lines cf(dir + "/init_configuration.dat");
    if (!cf.ok) return EDP_ERR_IO;
    double Te, Np;
    long long ncd, nmv, nbx, nby, ngx, ngy, nppc, cbx, cby, nbo, nio;
    bool good = true;
    good &= cf.next(L) && cf.next(L) && freal(L, 3, 12, &Te);
    good &= cf.next(L) && cf.next(L) && freal(L, 3, 14, &Np);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &ncd);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &nmv);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &nbx);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &nby);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &ngx);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &ngy);
    good &= cf.next(L) && cf.next(L) && fint(L, 2, 4, &nppc);
    good &= cf.next(L) && cf.next(L) && fint(L, 5, 1, &cbx);
    good &= cf.next(L) && cf.next(L) && fint(L, 5, 1, &cby);
    good &= cf.next(L) && cf.next(L) && fint(L, 3, 3, &nbo) && fint(L, 9, 3, &nio);
    if (!good || Te <= 0 || Np <= 0 || ncd < 1 || nmv < 1 || nbx < 1 || nby < 1 || ngx < 1 || ngy < 1 || nppc < 1)
        return EDP_ERR_IO;
    const int gmi = (int)(nbx * ngx + 1), gmj = (int)(nby * ngy + 1);   // global_maximal_i/j (:913-914)
    struct Seg { int is, js, ie, je; };
    std::vector<int> otype(nbo + nio);
    std::vector<std::vector<Seg>> osegs(nbo);
    for (int n = 0; n < nbo; ++n) {
        long long ty, ns;
        if (!(cf.next(L) && cf.next(L) && fint(L, 3, 2, &ty) && fint(L, 8, 2, &ns))) return EDP_ERR_IO;
        otype[n] = (int)ty;
        if (!cf.next(L)) return EDP_ERR_IO;
        for (int m = 0; m < ns; ++m) {
            long long a, b, c2, e;
            if (!(cf.next(L) && fint(L, 3, 6, &a) && fint(L, 12, 6, &b) && fint(L, 21, 6, &c2) && fint(L, 30, 6, &e)))
                return EDP_ERR_IO;
            osegs[n].push_back(Seg{(int)a, (int)b, (int)c2, (int)e});
        }
    }
    std::vector<Seg> inner(nio);
    for (int n = 0; n < nio; ++n) {
        long long ty, a, b, c2, e;
        if (!(cf.next(L) && cf.next(L) && fint(L, 3, 2, &ty))) return EDP_ERR_IO;
        if (!(cf.next(L) && cf.next(L) && fint(L, 3, 6, &a) && fint(L, 12, 6, &b) && fint(L, 21, 6, &c2) &&
              fint(L, 30, 6, &e)))
            return EDP_ERR_IO;
        otype[nbo + n] = (int)ty;
        inner[n] = Seg{(int)a, (int)b, (int)c2, (int)e};
    }
    // sides of the boundary objects
    int side_obj[4] = {-1, -1, -1, -1};   // below, above, left, right
    bool periodic_left = false, periodic_right = false;
    for (int n = 0; n < nbo; ++n)
        for (const Seg& s : osegs[n]) {
            int side = -1;
            if (s.js == s.je && s.js == 0) side = 0;
            else if (s.js == s.je && s.js == gmj) side = 1;
            else if (s.is == s.ie && s.is == 0) side = 2;
            else if (s.is == s.ie && s.is == gmi) side = 3;
            if (side < 0) continue;
            if (otype[n] == 2) {
                if (side == 2) periodic_left = true;
                if (side == 3) periodic_right = true;
                continue;
            }
            if (otype[n] != 1) return EDP_ERR_IO;   // dielectric / vacuum-gap walls are outside the supported subset
            side_obj[side] = n;
        }
    p.periodic_x = (periodic_left && periodic_right) ? 1 : 0;
    p.ncx = p.periodic_x ? gmi - 1 : gmi;
    p.ncy = gmj;
    p.n_of_particles_cell = (int32_t)nppc;
    // ---- scales (:719-723, :893-900)
    const double vte = std::sqrt(2.0 * Te * E_CL / M_E_KG);
    const double wp = std::sqrt(Np * (E_CL * E_CL) / (EPS0 * M_E_KG));   // N e**2 / (eps0 m)
    const double ld = vte / wp;
    p.delta_x_m = ld / ncd;
    p.delta_t_s = p.delta_x_m / (nmv * vte);
    p.v_scale_ms = nmv * vte;
    p.e_scale_vm = M_E_KG * p.v_scale_ms / (E_CL * p.delta_t_s);
    p.b_scale_t = M_E_KG / (E_CL * p.delta_t_s);
    p.f_scale_v = E_CL * Np * (p.delta_x_m * p.delta_x_m) / EPS0;   // e N dx**2 / eps0, in the reference's order
    d->t_e = Te;
    d->n_plasma = Np;
    d->n_max_vel = (int32_t)nmv;
    // ---- init_simcontrol.dat (:830-870)
    Lines sc(dir + "/init_simcontrol.dat");
    if (!sc.ok) return EDP_ERR_IO;
    double tsim;
    long long nsub;
    if (!(sc.next(L) && sc.next(L) && freal(L, 3, 11, &tsim) && sc.next(L) && sc.next(L) && fint(L, 8, 2, &nsub)))
        return EDP_ERR_IO;
    p.n_subcycles = (int32_t)nsub;
    d->max_t_cntr = (int64_t)(tsim / (1.0e9 * p.delta_t_s));
    // ---- init_particles.dat (:1005-1031)
    Lines pf(dir + "/init_particles.dat");
    if (!pf.ok) return EDP_ERR_IO;
    long long nspec, seed;
    if (!(pf.next(L) && pf.next(L) && freal(L, 3, 8, &d->init_te) && pf.next(L) && pf.next(L) &&
          freal(L, 3, 10, &d->init_ne) && pf.next(L) && pf.next(L) && fint(L, 6, 1, &nspec)))
        return EDP_ERR_IO;
    if (nspec < 1 || nspec > EDP_MAX_ION_SPECIES) return EDP_ERR_IO;
    p.n_ion_species = (int32_t)nspec;
    if (!pf.next(L)) return EDP_ERR_IO;
    for (int s = 0; s < nspec; ++s) {
        double m, ti, conc;
        long long q;
        if (!(pf.next(L) && freal(L, 3, 5, &m) && fint(L, 11, 2, &q) && freal(L, 16, 8, &ti) && freal(L, 27, 6, &conc)))
            return EDP_ERR_IO;
        p.ion_charge[s] = (int32_t)q;
        p.ion_mass_me[s] = (AMU_KG * m) / M_E_KG;
        d->init_ti[s] = ti;
    }
    if (!(pf.next(L) && pf.next(L) && fint(L, 3, 9, &seed))) return EDP_ERR_IO;
    p.seed = (uint64_t)seed;
    // ---- init_extfields.dat (pic2d_ExternalFields.f90:36-110)
    Lines ef(dir + "/init_extfields.dat");
    if (ef.ok) {
        double bx, by, yb, bz0, bzmax, bzl, h1, h2, ez;
        long long sb, se;
        bool g2 = ef.next(L) && ef.next(L) && freal(L, 3, 9, &bx) && ef.next(L) && ef.next(L) && freal(L, 3, 9, &by) &&
                  ef.next(L) && ef.next(L) && ef.next(L) && freal(L, 3, 9, &yb) && ef.next(L) && ef.next(L) &&
                  freal(L, 3, 9, &bz0) && ef.next(L) && ef.next(L) && freal(L, 3, 9, &bzmax) && ef.next(L) &&
                  ef.next(L) && freal(L, 3, 9, &bzl) && ef.next(L) && ef.next(L) && freal(L, 3, 9, &h1) &&
                  ef.next(L) && ef.next(L) && freal(L, 3, 9, &h2) && ef.next(L) && ef.next(L) &&
                  freal(L, 3, 9, &ez) && ef.next(L) && ef.next(L) && fint(L, 7, 1, &sb) && ef.next(L) &&
                  ef.next(L) && fint(L, 7, 1, &se);
        if (!g2) return EDP_ERR_IO;
        p.bx = bx * 1.0e-4 / p.b_scale_t;
        p.by = by * 1.0e-4 / p.b_scale_t;
        p.bz = bzmax * 1.0e-4 / p.b_scale_t;   // Bz_ext = Bz_max (:80)
        p.ez = ez * 100.0 / p.e_scale_vm;
        p.ions_sense_b = sb != 0;
        p.ions_sense_ez = se != 0;
    }
    // ---- init_bo_NN.dat (pic2d_Setup.f90:60-100) for metal walls and inner objects; normalised as :1218-1221
    auto read_bo = [&](int n, double* c0, double* var, double* om, double* ph) -> bool {
        char name[32];
        snprintf(name, sizeof(name), "/init_bo_%02d.dat", n + 1);
        Lines bf(dir + name);
        *c0 = *var = *om = *ph = 0.0;
        if (!bf.ok) return true;
        bool g3 = bf.next(L) && bf.next(L) && bf.next(L) && bf.next(L) && freal(L, 3, 9, c0) && bf.next(L) &&
                  bf.next(L) && freal(L, 3, 9, var) && bf.next(L) && bf.next(L) && freal(L, 3, 9, om) && bf.next(L) &&
                  bf.next(L) && freal(L, 3, 9, ph);
        *c0 /= p.f_scale_v;
        *var /= p.f_scale_v;
        *om = *om * 2.0e6 * PI * p.delta_t_s;
        *ph = *ph * PI / 180.0;
        return g3;
    };
    // the optional waveform and amplitude-profile files of a metal object (PREPARE_WAVEFORMS,
    // PREPARE_OSCILLATIONS_AMPLITUDE_PROFILE, pic2d_Setup.f90:150-412), named by the object's number
    auto read_profiles = [&](int n, EdpPotentialProfile* q) {
        char name[64];
        snprintf(name, sizeof(name), "/init_bo_%02d_waveform.dat", n + 1);
        edp_read_waveform(dir + name, p.delta_t_s, p.f_scale_v, q);
        snprintf(name, sizeof(name), "/init_bo_%02d_amplitude_profile.dat", n + 1);
        edp_read_amplitude_profile(dir + name, p.delta_t_s, q);
    };
    for (int s = 0; s < 4; ++s)
        if (side_obj[s] >= 0) {
            if (!read_bo(side_obj[s], &p.wall_phi_const[s], &p.wall_phi_var[s], &p.wall_omega[s], &p.wall_phase[s]))
                return EDP_ERR_IO;
            EdpPotentialProfile& q = d->pot[s];
            q.phi_const = p.wall_phi_const[s];
            q.phi_var = p.wall_phi_var[s];
            q.omega = p.wall_omega[s];
            q.phase = q.phase_adjusted = p.wall_phase[s];
            read_profiles(side_obj[s], &q);
        }
    // ---- constant electron emission of the walls (init_bo_NN.dat lines 11-20, PREPARE_SETUP_VALUES
    // pic2d_Setup.f90:86-95): macroparticles per step (3x,f9.3), model (7x,i1), normal and parallel temperatures and
    // the beam energy in eV (4x,f8.3)
    for (int w = 0; w < 4 + std::min<int>((int)nio, EDP_MAX_INNER); ++w) {
        const int bo = w < 4 ? side_obj[w] : (int)nbo + (w - 4);   // the walls, then the inner objects
        if (bo < 0) continue;
        char name[32];
        snprintf(name, sizeof(name), "/init_bo_%02d.dat", bo + 1);
        Lines bf(dir + name);
        if (!bf.ok) continue;
        for (int k = 0; k < 10; ++k)
            if (!bf.next(L)) return EDP_ERR_IO;
        long long model = 0;
        double* q = d->inject[w];
        bool ok = bf.next(L) && bf.next(L) && freal(L, 3, 9, &q[0]) && bf.next(L) && bf.next(L) &&
                  fint(L, 7, 1, &model) && bf.next(L) && bf.next(L) && freal(L, 4, 8, &q[2]) && bf.next(L) &&
                  bf.next(L) && freal(L, 4, 8, &q[3]) && bf.next(L) && bf.next(L) && freal(L, 4, 8, &q[4]);
        if (!ok) return EDP_ERR_IO;
        q[0] = (double)(float)q[0];   // N_electron_constant_emit is REAL
        q[1] = (double)model;
    }
    // ---- wall materials (material name: init_bo_NN.dat line 2, (6x,A6), pic2d_Setup.f90:77; properties
    // init_material_<NAME>.dat, PREPARE_WALL_MATERIALS pic2d_Materials.f90:1-200). Only the ion-material interaction
    // model is used: 2 = ion-induced electron emission with, per ion species, a constant coefficient between
    // E_min and E_max and the temperature of the emitted electrons. A missing file means default materials.
    for (int w = 0; w < 4 + std::min<int>((int)nio, EDP_MAX_INNER); ++w) {
        const int bo = w < 4 ? side_obj[w] : (int)nbo + (w - 4);   // the walls, then the inner objects
        if (bo < 0) continue;
        char name[32];
        snprintf(name, sizeof(name), "/init_bo_%02d.dat", bo + 1);
        Lines bf(dir + name);
        if (!bf.ok || !bf.next(L) || !bf.next(L)) continue;
        const std::string mat = (L + "      ").substr(6, 6);   // the six characters of the A6 field
        if (mat == "      ") continue;
        Lines mf(dir + "/init_material_" + mat + ".dat");
        if (!mf.ok) continue;
        {
            // lines 3-56, in the order of pic2d_Materials.f90:84-149 (one header line before each value)
            Lines sf(dir + "/init_material_" + mat + ".dat");
            edp_see_params& s = d->see[w];
            long long m1 = 0, rt = 0, m2 = 0, m3 = 0;
            auto I = [&](long long* v) { return sf.next(L) && sf.next(L) && fint(L, 7, 1, v); };
            auto R = [&](size_t skip, size_t width, double* v) { return sf.next(L) && sf.next(L) && freal(L, skip, width, v); };
            auto H = [&]() { return sf.next(L); };
            double eps = 0;
            bool ok = R(6, 6, &eps) && I(&m1) && I(&rt) && H() && R(7, 5, &s.elastic_yield) &&
                      R(2, 10, &s.elastic_emin_ev) && R(2, 10, &s.elastic_emax_ev) && H() && R(2, 10, &s.elastic_e0_ev) &&
                      R(2, 10, &s.elastic_emax_coef_ev) && R(7, 5, &s.elastic_max) && R(2, 10, &s.elastic_de_ev) &&
                      R(7, 5, &s.elastic_frac_classic) && I(&m2) && H() && R(7, 5, &s.inelastic_yield) &&
                      R(2, 10, &s.inelastic_emin_ev) && R(2, 10, &s.inelastic_emax_ev) && H() &&
                      R(7, 5, &s.inelastic_frac_classic) && I(&m3) && R(2, 10, &s.true_t_ev) && H() &&
                      R(7, 5, &s.true_yield) && R(2, 10, &s.true_emin_ev) && R(2, 10, &s.true_emax_ev) && H() &&
                      R(2, 10, &s.classic_e0_ev) && R(2, 10, &s.classic_emax_ev) && R(6, 6, &s.classic_max) &&
                      R(7, 5, &s.classic_k_smooth);
            if (!ok) return EDP_ERR_IO;
            s.elastic_model = (int32_t)m1;
            s.elastic_type = (int32_t)rt;
            s.inelastic_model = (int32_t)m2;
            s.true_model = (int32_t)m3;
        }
        bool found = false;
        while (mf.next(L))
            if (L.find("ION-MATERIAL INTERACTION MODEL") != std::string::npos) {
                found = true;
                break;
            }
        long long flag = 0;
        if (!found || !mf.next(L) || !fint(L, 7, 1, &flag)) continue;
        flag = std::max(0LL, std::min(flag, 2LL));   // MAX(0, MIN(flag, 2)), :153
        d->ion_model[w] = (int32_t)flag;
        if (flag != 2) continue;
        for (int s = 0; s < (int)p.n_ion_species; ++s) {
            double yv = 0, e0 = 0, e1 = 0, te = 0;
            bool ok = mf.next(L) && mf.next(L) && mf.next(L) && freal(L, 7, 5, &yv) && mf.next(L) && mf.next(L) &&
                      freal(L, 2, 10, &e0) && mf.next(L) && mf.next(L) && freal(L, 2, 10, &e1) && mf.next(L) &&
                      mf.next(L) && freal(L, 2, 10, &te);
            if (!ok) return EDP_ERR_IO;
            d->ii_ee[w][s][0] = yv;
            d->ii_ee[w][s][1] = e0;
            d->ii_ee[w][s][2] = e1;
            d->ii_ee[w][s][3] = te;
        }
    }
    if (nio > EDP_MAX_INNER) return EDP_ERR_IO;
    p.n_inner = (int32_t)nio;
    for (int n = 0; n < nio; ++n) {
        // METAL_WALL = 1 or DIELECTRIC = 4 (pic2d_Modules.f90:143-147); a dielectric's permittivity is the first
        // value of its material file, (6x,f6.3) (pic2d_Materials.f90:81-82)
        if (otype[nbo + n] != 1 && otype[nbo + n] != 4) return EDP_ERR_IO;
        p.inner_eps[n] = 0.0;
        if (otype[nbo + n] == 4) {
            if (p.periodic_x) return EDP_ERR_IO;   // dielectrics: CG solver (walled domain) only
            char name[32];
            snprintf(name, sizeof(name), "/init_bo_%02d.dat", (int)(nbo + n + 1));
            Lines bf(dir + name);
            if (!bf.ok || !bf.next(L) || !bf.next(L)) return EDP_ERR_IO;
            const std::string mat = (L + "      ").substr(6, 6);
            Lines mf(dir + "/init_material_" + mat + ".dat");
            double eps = 0.0;
            if (!mf.ok || !mf.next(L) || !mf.next(L) || !freal(L, 6, 6, &eps) || !(eps > 0.0)) return EDP_ERR_IO;
            p.inner_eps[n] = eps;
        }
        p.inner_ileft[n] = inner[n].is;
        p.inner_jbottom[n] = inner[n].js;
        p.inner_iright[n] = inner[n].ie;
        p.inner_jtop[n] = inner[n].je;
        double c0, var, om, ph;
        if (!read_bo(nbo + n, &c0, &var, &om, &ph)) return EDP_ERR_IO;
        EdpPotentialProfile& q = d->pot[4 + n];
        q.phi_const = c0;
        q.phi_var = var;
        q.omega = om;
        q.phase = q.phase_adjusted = ph;
        if (otype[nbo + n] == 1) read_profiles(nbo + n, &q);   // METAL_WALL only
        EdpPotentialProfile q0 = q;
        p.inner_phi[n] = q0.value(0);   // UPDATE_WALL_POTENTIALS(0) at set-up (pic2d_CurProblemValues.f90:1226)
    }
    p.precision = EDP_PREC_MIXED;
    p.solver = p.periodic_x ? EDP_SOLVER_FFTX : EDP_SOLVER_CG;
    p.sort_every = 80;   // order does not change results (fixed-point deposit); 80 measured fastest at cfg1
    p.fuse_collisions = 1;
    // ---- Maxwell table (PrepareMaxwellDistribIntegral, pic2d_ElectronWallCollisions.f90:835-929)
    {
        const int N = 180000, R = 9000;
        const double vmin = -3.0, dv = 6.0 / N;
        std::vector<double> F(N + 4, 0.0);
        for (int i = 1; i <= N + 3; ++i) {
            double u = vmin + ((double)i - 0.5) * dv;
            F[i] = F[i - 1] + std::exp(-(u * u));
        }
        double tot = F[N];
        d->maxwell.assign(R + 1, 0.0);
        d->maxwell[0] = vmin;
        int count = 0;
        for (int i = 1; i <= N + 3 && count < R; ++i) {
            if ((int)(F[i] * R / tot) - count == 1) d->maxwell[++count] = vmin + i * dv;
        }
        t.maxwell_rmax = R;
        t.maxwell_v = d->maxwell.data();
    }
    t.energy_factor_eV = 0.5 * M_E_KG * (p.v_scale_ms * p.v_scale_ms) / E_CL;
    // ---- neutrals (pic2d_enCollisionsGeneralProc.f90:63-200)
    Lines nf(dir + "/init_neutrals.dat");
    if (!nf.ok) return EDP_OK;   // no neutrals: collisions off
    long long nneu;
    if (!(nf.next(L) && nf.next(L) && fint(L, 10, 2, &nneu))) return EDP_ERR_IO;
    if (nneu <= 0) return EDP_OK;
    if (nneu > 1) return EDP_ERR_IO;
    std::string name;
    double ngas, tgas;
    if (!(nf.next(L) && nf.next(L))) return EDP_ERR_IO;
    name = L.size() > 6 ? L.substr(6, 6) : "";
    if (!(nf.next(L) && nf.next(L) && freal(L, 2, 10, &ngas) && nf.next(L) && nf.next(L) && freal(L, 5, 7, &tgas)))
        return EDP_ERR_IO;
    Lines nn(dir + "/init_neutral_" + name + ".dat");
    std::vector<CrossSection> procs;
    double mass = 0;
    if (nn.ok) {
        long long ncp;
        if (!(nn.next(L) && nn.next(L) && freal(L, 3, 7, &mass) && nn.next(L) && nn.next(L) && fint(L, 8, 2, &ncp)))
            return EDP_ERR_IO;
        for (int q = 0; q < ncp; ++q) {
            CrossSection cs;
            long long ty, act, isp, sv;
            if (!(nn.next(L) && nn.next(L) && fint(L, 3, 2, &ty) && fint(L, 7, 1, &act) && fint(L, 10, 2, &isp) &&
                  fint(L, 14, 1, &sv)))
                return EDP_ERR_IO;
            cs.type = (int)ty;
            cs.activated = act != 0;
            cs.ion_species = (int)isp;
            procs.push_back(cs);
        }
        long long nseg;
        if (!(nn.next(L) && nn.next(L) && fint(L, 8, 2, &nseg))) return EDP_ERR_IO;
        if (nseg < 1 || nseg > EDP_MAX_SEGMENTS) return EDP_ERR_IO;
        t.n_seg = (int32_t)nseg;
        if (!(nn.next(L) && nn.next(L) && freal(L, 2, 9, &t.seg_value[0]))) return EDP_ERR_IO;
        for (int i = 1; i <= nseg; ++i)
            if (!(nn.next(L) && nn.next(L) && freal(L, 2, 9, &t.seg_value[i]) && freal(L, 14, 7, &t.seg_step[i - 1])))
                return EDP_ERR_IO;
        // cross sections of the activated processes (:170-200)
        for (size_t q = 0; q < procs.size(); ++q) {
            if (!procs[q].activated) continue;
            char fn[96];
            snprintf(fn, sizeof(fn), "/init_neutral_%s_crsect_coll_id_%02d_type_%02d.dat", name.c_str(), (int)q + 1,
                     procs[q].type);
            Lines xf(dir + fn);
            long long np;
            if (!(xf.ok && xf.next(L) && fint(L, 2, 4, &np)) || np < 2) return EDP_ERR_IO;
            for (int k = 0; k < np; ++k) {
                double e, s;
                if (!(xf.next(L) && freal(L, 4, 9, &e) && freal(L, 15, 10, &s))) return EDP_ERR_IO;
                procs[q].e.push_back(e);
                procs[q].s.push_back(s);
            }
        }
    }
    std::vector<const CrossSection*> act;
    for (auto& q : procs)
        if (q.activated) act.push_back(&q);
    if (!act.empty()) {
        if (act.size() > EDP_MAX_COLPROC) return EDP_ERR_IO;
        t.en_on = 1;
        t.n_act = (int32_t)act.size();
        t.neutral_mass_amu = mass;
        // energy grid and probability table (:236-322)
        int nv = 0;
        for (int i = 1; i <= t.n_seg; ++i) nv += (int)((t.seg_value[i] - t.seg_value[i - 1]) / t.seg_step[i - 1] + 0.001);
        t.n_values = nv;
        t.seg_index[0] = 0;
        for (int i = 1; i <= t.n_seg; ++i)
            t.seg_index[i] = t.seg_index[i - 1] + (int)((t.seg_value[i] - t.seg_value[i - 1]) / t.seg_step[i - 1] + 0.001);
        d->energy.assign(nv + 1, 0.0);
        d->energy[0] = t.seg_value[0];
        for (int i = 1; i <= t.n_seg; ++i) {
            for (int j = t.seg_index[i - 1] + 1; j <= t.seg_index[i] - 1; ++j)
                d->energy[j] = t.seg_value[i - 1] + (j - t.seg_index[i - 1]) * t.seg_step[i - 1];
            d->energy[t.seg_index[i]] = t.seg_value[i];
        }
        const int na = t.n_act;
        d->prob.assign((size_t)(nv + 1) * na, 0.0);
        for (int ie = 0; ie <= nv; ++ie) {
            double run = 0.0;
            for (int q = 0; q < na; ++q) {
                run = (q == 0 ? 0.0 : run) + en_frequency(*act[q], d->energy[ie], ngas, p.n_subcycles, p.delta_t_s);
                d->prob[(size_t)ie * na + q] = run;
            }
        }
        int imax = 0;
        for (int ie = 1; ie <= nv; ++ie)
            if (d->prob[(size_t)ie * na + na - 1] > d->prob[(size_t)imax * na + na - 1]) imax = ie;
        const double pm = d->prob[(size_t)imax * na + na - 1];
        t.max_colliding_fraction = 1.0 - std::exp(-pm);
        for (auto& v : d->prob) v = std::fmax(0.0, std::fmin(1.0, v / pm));
        d->prob[(size_t)imax * na + na - 1] = 1.0;
        for (int ie = 0; ie <= nv; ++ie)
            for (int q = 0; q + 1 < na; ++q)
                d->prob[(size_t)ie * na + q + 1] = std::fmax(d->prob[(size_t)ie * na + q], d->prob[(size_t)ie * na + q + 1]);
        for (int q = 0; q < na; ++q) {
            t.colproc_type[q] = act[q]->type;
            t.threshold_eV[q] = act[q]->type >= 20 ? act[q]->e[0] : 0.0;
            t.ion_species_produced[q] = act[q]->ion_species;
            int s = act[q]->ion_species;
            if (s >= 1 && s <= nspec)
                t.ion_velocity_factor[q] = std::sqrt(tgas * KB_JK / (Te * E_CL)) / (nmv * std::sqrt(p.ion_mass_me[s - 1]));
        }
        t.prob = d->prob.data();
        t.energy_eV = d->energy.data();
    }
    // ---- resonant charge exchange (pic2d_inCollisionsGeneralProc.f90:50-90, pic2d_inCollisionsSpecificProc.f90:4-31)
    std::ifstream rf(dir + "/init_neutral_" + name + "_rcx_param.dat");
    if (rf) {
        std::string hdr;
        std::getline(rf, hdr);
        long long s;
        double sig, alpha;
        if (!(rf >> s >> sig >> alpha)) return EDP_ERR_IO;
        if (s >= 1 && s <= nspec) {
            int k = (int)s - 1;
            t.rcx_on[k] = 1;
            t.rcx_sigma_1eV = sig;
            t.rcx_alpha = alpha;
            t.rcx_prob_factor = ngas * p.delta_t_s * p.n_subcycles;
            t.rcx_vfactor[k] = std::sqrt(tgas * KB_JK / (Te * E_CL * p.ion_mass_me[k])) / (double)nmv;
            double tg_eV = tgas * KB_JK / E_CL;
            double l = 1.0 - alpha * std::log(std::fmax(1.5 * tg_eV, 0.001));
            double sth = sig * (l * l);
            double vmean = std::sqrt(2.54647908947033 * tg_eV * E_CL / (p.ion_mass_me[k] * M_E_KG));
            t.rcx_probab_thermal[k] = ngas * sth * vmean * p.delta_t_s * p.n_subcycles;
        }
    }
    return EDP_OK;
}

}  // namespace

extern "C" {

int edp_deck_read(const char* dir, edp_deck** out, edp_params* p, edp_tables* t)
{
    if (!dir || !out || !p || !t) return EDP_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<edp_deck> d(new edp_deck());
    int r = read_deck(dir, d.get());
    if (r != EDP_OK) return r;
    *p = d->p;
    *t = d->t;
    *out = d.release();
    return EDP_OK;
}

int edp_deck_initial_plasma(const edp_deck* d, double* te, double* ne, double* ti, double* t_e, int32_t* nmv,
                            double* np, int64_t* maxt)
{
    if (!d) return EDP_ERR_ARG;
    if (te) *te = d->init_te;
    if (ne) *ne = d->init_ne;
    if (ti)
        for (int s = 0; s < EDP_MAX_ION_SPECIES; ++s) ti[s] = d->init_ti[s];
    if (t_e) *t_e = d->t_e;
    if (nmv) *nmv = d->n_max_vel;
    if (np) *np = d->n_plasma;
    if (maxt) *maxt = d->max_t_cntr;
    return EDP_OK;
}

int edp_deck_ion_emission(const edp_deck* d, int32_t wall, int32_t ion_species, double* out)
{
    if (!d || !out || wall < 0 || wall >= EDP_N_HIT_COUNTERS || ion_species < 1 || ion_species > EDP_MAX_ION_SPECIES)
        return EDP_ERR_ARG;
    for (int k = 0; k < 4; ++k) out[k] = d->ii_ee[wall][ion_species - 1][k];
    return EDP_OK;
}

int edp_deck_ion_wall_model(const edp_deck* d, int32_t wall, int32_t* model)
{
    if (!d || !model || wall < 0 || wall >= EDP_N_HIT_COUNTERS) return EDP_ERR_ARG;
    *model = d->ion_model[wall];
    return EDP_OK;
}

int edp_deck_electron_emission(const edp_deck* d, int32_t wall, edp_see_params* out, int32_t* enabled)
{
    if (!d || !out || wall < 0 || wall >= EDP_N_HIT_COUNTERS) return EDP_ERR_ARG;
    *out = d->see[wall];
    if (enabled) *enabled = (out->elastic_model + out->inelastic_model + out->true_model) > 0;
    return EDP_OK;
}

int edp_deck_wall_injection(const edp_deck* d, int32_t wall, double* out)
{
    if (!d || !out || wall < 0 || wall >= EDP_N_HIT_COUNTERS) return EDP_ERR_ARG;
    for (int k = 0; k < 5; ++k) out[k] = d->inject[wall][k];
    return EDP_OK;
}

int edp_deck_potential_profile(const edp_deck* d, int32_t object, double* harmonic, int32_t* n_wf, int32_t* wf_t,
                               float* wf_phi, int32_t* n_ap, int32_t* ap_t, float* ap_factor)
{
    if (!d || object < 0 || object >= 4 + EDP_MAX_INNER || !n_wf || !n_ap) return EDP_ERR_ARG;
    const EdpPotentialProfile& q = d->pot[object];
    if (harmonic) {
        harmonic[0] = q.phi_const;
        harmonic[1] = q.phi_var;
        harmonic[2] = q.omega;
        harmonic[3] = q.phase;
    }
    *n_wf = (int32_t)q.wf_t.size();
    *n_ap = (int32_t)q.ap_t.size();
    for (size_t k = 0; k < q.wf_t.size(); ++k) {
        if (wf_t) wf_t[k] = q.wf_t[k];
        if (wf_phi) wf_phi[k] = q.wf_phi[k];
    }
    for (size_t k = 0; k < q.ap_t.size(); ++k) {
        if (ap_t) ap_t[k] = q.ap_t[k];
        if (ap_factor) ap_factor[k] = q.ap_factor[k];
    }
    return EDP_OK;
}

int edp_deck_potential_series(const edp_deck* d, int32_t object, int64_t t0, int64_t n, double* out)
{
    if (!d || object < 0 || object >= 4 + EDP_MAX_INNER || t0 < 0 || n < 0 || t0 + n > INT32_MAX || (n && !out))
        return EDP_ERR_ARG;
    EdpPotentialProfile q = d->pot[object];
    q.adjust_phase((int32_t)t0);
    for (int64_t k = 0; k < n; ++k) out[k] = q.value((int32_t)(t0 + k));
    return EDP_OK;
}

int edp_deck_free(edp_deck* d)
{
    delete d;
    return EDP_OK;
}

}  // extern "C"

// C entry points over the reference library, compiled from the reference's own
// sources (oracle/Makefile).  Test infrastructure only: the tests, smoke() and
// the CPU-baseline leg of bench.py load this to pin the oracle restatement and
// to time the reference CPU path.  Nothing in the product links it.
//
// Every function here forwards to the reference's public API unchanged:
//   bblock::System setup            bblock/system.h:564 (AddMonomer),
//                                    :578 (AddMolecule), :713 (Initialize),
//                                    :776 (SetUpFromJson)
//   TwoBodyEnergy / ThreeBodyEnergy  bblock/system.h:1088, :1100
//   GetRealGrads / GetVirial         bblock/system.h:285, :450
//   GetPairList                      bblock/system.h:246
//   e2b::get_2b_energy               potential/2b/energy2b.h:109
//   e3b::get_3b_energy               potential/3b/energy3b.h:102
//   generated polynomials            potential/2b/poly-2b-v6x.h:78,95;
//                                    potential/3b/poly-3b-v2x.h:73,86; ...
#include <cstring>
#include <sstream>
#include <string>
#include <vector>
#include <exception>
#include <cstdio>
#include <cstdlib>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "bblock/system.h"
#include "potential/2b/energy2b.h"
#include "potential/3b/energy3b.h"
#include "potential/2b/poly-2b-v6x.h"
#include "potential/3b/poly-3b-v2x.h"
#include "potential/2b/poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x.h"
#include "potential/2b/poly_2b_A1B4_A1B4_deg4_exp0_v1x.h"
#include "potential/3b/poly_3b_A1B4_C1D2_C1D2_deg3_v1.h"
#include "potential/2b/poly-2b-A1B2Z2_C-v1x.h"
#include "potential/3b/poly-3b-h2o-ion-v1x_deg4_filtered.h"
#include "potential/2b/poly_2b_A1_B1C2X2_deg6_v1.h"
#include "potential/3b/poly_3b_A1_B1C2X2_B1C2X2_deg4_v1.h"
#include "potential/2b/poly_2b_A1_A1_deg9_v1.h"
#include "potential/2b/poly_2b_A1_B1_deg9_v1.h"
#include "potential/2b/poly_2b_A1_B1C2X2_deg5_v1.h"
#include "potential/2b/poly_2b_A1B2_A1B2_v1x.h"
#include "potential/2b/poly_2b_A1B2Z2_C1D2_v1x.h"
#include "potential/2b/poly_2b_A1_A1_deg23_v1x.h"
#include "potential/2b/poly_2b_A1B2Z2_C1_deg5_v1x.h"
#include "potential/2b/poly_2b_A2_A2_deg6_v1.h"
#include "potential/2b/poly_2b_A1B2Z2_C2_deg5_v1.h"
#include "potential/2b/poly_2b_A1_B2_deg7_v1.h"
#include "potential/2b/poly_2b_A1B3_A1B3_deg4_v1.h"
#include "potential/2b/poly_2b_A1B4_C1D2_deg4_v1.h"
#include "potential/2b/poly_2b_A1B2Z2_A1B2Z2_deg4_vmbpbe.h"
#include "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_v1.h"
#include "potential/3b/poly_3b_A1B2_A1B2_A1B2_deg4_vmbpbe.h"
#include "potential/2b/poly_2b_A1B2C4_D1E2_deg3_v1x.h"
#include "potential/3b/poly_3b_A1B2C4_D1E2_D1E2_deg3_v1.h"

namespace {

thread_local std::string g_err;

std::vector<std::string> split_ids(const char* ids) {
    std::vector<std::string> out;
    std::istringstream iss(ids);
    std::string w;
    while (iss >> w) out.push_back(w);
    return out;
}

std::vector<std::string> atom_names(const std::string& id) {
    if (id == "h2o") return {"O", "H", "H"};
    if (id == "ch4") return {"C", "H", "H", "H", "H"};
    if (id == "li+") return {"Li"};
    if (id == "na+") return {"Na"};
    if (id == "k+") return {"K"};
    if (id == "rb+") return {"Rb"};
    if (id == "cs+") return {"Cs"};
    if (id == "f-") return {"F"};
    if (id == "cl-") return {"Cl"};
    if (id == "br-") return {"Br"};
    if (id == "i-") return {"I"};
    if (id == "ar") return {"Ar"};
    if (id == "h2") return {"H", "H"};
    if (id == "nh3" || id == "nh3pbe0d3bj") return {"N", "H", "H", "H"};
    if (id == "co2" || id == "co2_archive" || id.rfind("co2cm", 0) == 0) return {"C", "O", "O"};
    if (id == "mbpbe") return {"O", "H", "H"};
    if (id == "he") return {"He"};
    if (id == "n2o5") return {"O", "N", "N", "O", "O", "O", "O"};
    throw std::runtime_error("harness knows no atom names for monomer id " + id);
}

}  // namespace

extern "C" {

const char* mbxref_last_error() { return g_err.c_str(); }

void mbxref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int mbxref_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// ids: whitespace-separated monomer ids in input order; xyz: real-atom
// coordinates in input order (3 doubles per atom); json: the "MBX" config text.
void* mbxref_new(const char* ids, const double* xyz, const char* json) {
    try {
        auto* sys = new bblock::System();
        std::vector<std::string> mons = split_ids(ids);
        size_t off = 0;
        for (size_t m = 0; m < mons.size(); ++m) {
            std::vector<std::string> names = atom_names(mons[m]);
            std::vector<double> x(xyz + 3 * off, xyz + 3 * (off + names.size()));
            sys->AddMonomer(x, names, mons[m]);
            sys->AddMolecule({m});
            off += names.size();
        }
        sys->Initialize();
        sys->SetUpFromJson(std::string(json));
        return sys;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// Defined only in the build whose System forwards its 2b/3b terms to the
// GPU library (ref_gpu_glue.cpp): releases that System's library context.
void mbxref_gpu_release(const void* sys) __attribute__((weak));

void mbxref_free(void* h) {
    if (mbxref_gpu_release) mbxref_gpu_release(h);
    delete static_cast<bblock::System*>(h);
}

int mbxref_set_real_xyz(void* h, const double* xyz) {
    try {
        auto* sys = static_cast<bblock::System*>(h);
        std::vector<double> x(xyz, xyz + 3 * sys->GetNumRealSites());
        sys->SetRealXyz(x);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int mbxref_num_real_sites(void* h) { return (int)static_cast<bblock::System*>(h)->GetNumRealSites(); }

// nbody = 2 or 3.  Returns 0 on success; energy in *e.
int mbxref_energy(void* h, int nbody, int do_grads, double* e) {
    try {
        auto* sys = static_cast<bblock::System*>(h);
        *e = nbody == 1   ? sys->OneBodyEnergy(do_grads != 0)
             : nbody == 2 ? sys->TwoBodyEnergy(do_grads != 0)
                          : sys->ThreeBodyEnergy(do_grads != 0);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Gradients of the real atoms, input order (3 doubles per atom).
void mbxref_real_grads(void* h, double* out) {
    std::vector<double> g = static_cast<bblock::System*>(h)->GetRealGrads();
    std::memcpy(out, g.data(), g.size() * sizeof(double));
}

void mbxref_virial(void* h, double* out9) {
    std::vector<double> v = static_cast<bblock::System*>(h)->GetVirial();
    for (int k = 0; k < 9; ++k) out9[k] = v[k];
}

// n-mer list in input monomer order.  Writes up to cap indices, returns the
// total number of indices (nmax * number of n-mers), or -1 on error.
long mbxref_pair_list(void* h, int nmax, double cutoff, unsigned long* out, long cap) {
    try {
        auto* sys = static_cast<bblock::System*>(h);
        std::vector<size_t> p = sys->GetPairList(nmax, cutoff, 0, sys->GetNumMon());
        long n = (long)p.size();
        for (long i = 0; i < n && i < cap; ++i) out[i] = p[i];
        return n;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Term dispatch, batch of nm n-mers of one type tuple (A8/A9).
double mbxref_get_2b(const char* m1, const char* m2, long nm, const double* xyz1, const double* xyz2,
                     long n1, long n2, double* g1, double* g2, double* virial9) {
    std::vector<double> x1(xyz1, xyz1 + n1), x2(xyz2, xyz2 + n2);
    std::vector<double> gg1(g1, g1 + n1), gg2(g2, g2 + n2), vir(virial9, virial9 + 9);
    double e = e2b::get_2b_energy(m1, m2, nm, x1, x2, gg1, gg2, &vir);
    std::memcpy(g1, gg1.data(), n1 * sizeof(double));
    std::memcpy(g2, gg2.data(), n2 * sizeof(double));
    for (int k = 0; k < 9; ++k) virial9[k] = vir[k];
    return e;
}

double mbxref_get_3b(const char* m1, const char* m2, const char* m3, long nm, const double* xyz1,
                     const double* xyz2, const double* xyz3, long n1, long n2, long n3, double* g1, double* g2,
                     double* g3, double* virial9) {
    std::vector<double> x1(xyz1, xyz1 + n1), x2(xyz2, xyz2 + n2), x3(xyz3, xyz3 + n3);
    std::vector<double> gg1(g1, g1 + n1), gg2(g2, g2 + n2), gg3(g3, g3 + n3), vir(virial9, virial9 + 9);
    double e = e3b::get_3b_energy(m1, m2, m3, nm, x1, x2, x3, gg1, gg2, gg3, &vir);
    std::memcpy(g1, gg1.data(), n1 * sizeof(double));
    std::memcpy(g2, gg2.data(), n2 * sizeof(double));
    std::memcpy(g3, gg3.data(), n3 * sizeof(double));
    for (int k = 0; k < 9; ++k) virial9[k] = vir[k];
    return e;
}

// Raw generated polynomials.  kind: 0 MB-pol 2b (31 vars), 1 MB-pol 3b (36),
// 2 CH4-H2O 2b (38), 3 CH4-CH4 2b (45), 4 CH4-H2O-H2O 3b (55), 5 alkali-ion -
// water 2b (8), 6 water - water - alkali-ion 3b (21), 7 halide - water 2b (8),
// 8 halide - water - water 3b (41), 9 like atoms 2b (1), 10 unlike atoms 2b (1),
// 11 argon - water 2b (8); 12-19 the template MB-nrg tables h2h22b, h2oh22b,
// csh22b, nh3nh32b, ch4co22b, mbpbe2b, co23b, mbpbe3b; 20 CO2 - CO2 2b (15),
// 21 H2O - CO2 2b (21), 22 He - He 2b (1), 23 H2O - He 2b (8), 24 N2O5 - H2O
// 2b (45), 25 N2O5 - H2O - H2O 3b (78).
// One configuration per call; g may be NULL for energy only.
double mbxref_poly(int kind, const double* a, const double* x, double* g) {
    switch (kind) {
        case 0: {
            if (!g) return x2o::poly_2b_v6x::eval(1, a, x)[0];
            alignas(128) static thread_local double t[3200 * 8];
            return x2o::poly_2b_v6x::eval(1, a, x, t, g)[0];
        }
        case 1: {
            if (!g) return x2o::poly_3b_v2x::eval(a, x);
            // lane-major [36][8]; evaluate lane 0 with the other lanes zeroed
            alignas(128) static thread_local double t[3500 * 8];
            double xl[36 * 8] = {0}, gl[36 * 8] = {0};
            for (int j = 0; j < 36; ++j) xl[j * 8] = x[j];
            double* e = x2o::poly_3b_v2x::eval(a, xl, t, gl);
            double r = e[0];
            delete[] e;
            for (int j = 0; j < 36; ++j) g[j] = gl[j * 8];
            return r;
        }
        case 2:
            return g ? x2b_A1B2Z2_C1D4_deg3_exp0::poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x::eval(a, x, g)
                     : x2b_A1B2Z2_C1D4_deg3_exp0::poly_2b_A1B2Z2_C1D4_deg3_exp0_v1x::eval(a, x);
        case 3:
            return g ? x2b_A1B4_A1B4_deg4_exp0::poly_2b_A1B4_A1B4_deg4_exp0_v1x::eval(a, x, g)
                     : x2b_A1B4_A1B4_deg4_exp0::poly_2b_A1B4_A1B4_deg4_exp0_v1x::eval(a, x);
        case 4: {
            mbnrg_A1B4_C1D2_C1D2_deg3::poly_A1B4_C1D2_C1D2_deg3_v1 p;
            return g ? p.eval(x, a, g) : p.eval(x, a);
        }
        case 5: {
            if (!g) return h2o_ion::poly_2b_h2o_ion_v1x::eval(1, a, x)[0];
            for (int j = 0; j < 8; ++j) g[j] = 0.0;
            return h2o_ion::poly_2b_h2o_ion_v1x::eval(1, a, x, g)[0];
        }
        case 6: {
            double gs[21];
            return h2o_ion::poly_3b_h2o_ion_v1x_deg4_filtered::eval(a, x, g ? g : gs);
        }
        case 7: {
            mbnrg_A1_B1C2X2_deg6::poly_A1_B1C2X2_deg6_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 8; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 8: {
            mbnrg_A1_B1C2X2_B1C2X2_deg4::poly_A1_B1C2X2_B1C2X2_deg4_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 41; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 9: {
            mbnrg_A1_A1_deg9::poly_A1_A1_deg9_v1 p;
            if (!g) return p.eval(x, a);
            g[0] = 0.0;
            return p.eval(x, a, g);
        }
        case 10: {
            mbnrg_A1_B1_deg9::poly_A1_B1_deg9_v1 p;
            if (!g) return p.eval(x, a);
            g[0] = 0.0;
            return p.eval(x, a, g);
        }
        case 11: {
            mbnrg_A1_B1C2X2_deg5::poly_A1_B1C2X2_deg5_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 8; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 12: {
            mbnrg_A2_A2_deg6::poly_A2_A2_deg6_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 6; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 13: {
            mbnrg_A1B2Z2_C2_deg5::poly_A1B2Z2_C2_deg5_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 14; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 14: {
            mbnrg_A1_B2_deg7::poly_A1_B2_deg7_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 3; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 15: {
            mbnrg_A1B3_A1B3_deg4::poly_A1B3_A1B3_deg4_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 28; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 16: {
            mbnrg_A1B4_C1D2_deg4::poly_A1B4_C1D2_deg4_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 28; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 17: {
            mbnrg_A1B2Z2_A1B2Z2_deg4::poly_A1B2Z2_A1B2Z2_deg4_vmbpbe p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 31; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 18: {
            mbnrg_A1B2_A1B2_A1B2_deg4::poly_A1B2_A1B2_A1B2_deg4_v1 p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 27; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
        case 19: {
            mbnrg_A1B2_A1B2_A1B2_deg4::poly_A1B2_A1B2_A1B2_deg4_vmbpbe p;
            if (!g) return p.eval(x, a);
            for (int j = 0; j < 36; ++j) g[j] = 0.0;
            return p.eval(x, a, g);
        }
    }
    if (kind == 20) {
        if (!g) return x2b_A1B2_A1B2_deg5::poly_2b_A1B2_A1B2_deg5_v1x::eval(a, x);
        for (int j = 0; j < 15; ++j) g[j] = 0.0;
        return x2b_A1B2_A1B2_deg5::poly_2b_A1B2_A1B2_deg5_v1x::eval(a, x, g);
    }
    if (kind == 22 || kind == 23) {
        const int nv = kind == 22 ? 1 : 8;
        if (g)
            for (int j = 0; j < nv; ++j) g[j] = 0.0;
        if (kind == 22) return g ? x2b_A1_A1_deg23::poly_2b_A1_A1_deg23_v1x::eval(a, x, g)
                                 : x2b_A1_A1_deg23::poly_2b_A1_A1_deg23_v1x::eval(a, x);
        return g ? x2b_A1B2Z2_C1_deg5::poly_2b_A1B2Z2_C1_deg5_v1x::eval(a, x, g)
                 : x2b_A1B2Z2_C1_deg5::poly_2b_A1B2Z2_C1_deg5_v1x::eval(a, x);
    }
    if (kind == 24) {
        if (!g) return x2b_A1B2C4_D1E2_deg3::poly_2b_A1B2C4_D1E2_deg3_v1x::eval(a, x);
        for (int j = 0; j < 45; ++j) g[j] = 0.0;
        return x2b_A1B2C4_D1E2_deg3::poly_2b_A1B2C4_D1E2_deg3_v1x::eval(a, x, g);
    }
    if (kind == 25) {
        mbnrg_A1B2C4_D1E2_D1E2_deg3::poly_A1B2C4_D1E2_D1E2_deg3_v1 p;
        if (!g) return p.eval(x, a);
        for (int j = 0; j < 78; ++j) g[j] = 0.0;
        return p.eval(x, a, g);
    }
    if (kind == 21) {
        if (!g) return x2b_A1B2Z2_C1D2_deg4::poly_2b_A1B2Z2_C1D2_deg4_v1x::eval(a, x);
        for (int j = 0; j < 21; ++j) g[j] = 0.0;
        return x2b_A1B2Z2_C1D2_deg4::poly_2b_A1B2Z2_C1D2_deg4_v1x::eval(a, x, g);
    }
    return 0.0;
}

}  // extern "C"

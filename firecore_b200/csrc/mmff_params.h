// mmff_params.h -- this project's element x hybridisation parameter table,
// shared by the synthetic generator (molgen.cpp) and the xyz topology builder
// of the legacy interface (mmff_legacy.cpp).
//
// Meaning of the values follows MM::Builder::toMMFFsp3_loc
// (cpp/common/molecular/MMFFBuilder.h:4153-4300): rest angles by
// hybridisation, apars = (cos(a0/2), sin(a0/2), 4*Kss, sin(Asp)), bond k/l0
// per element pair, Ksp on nodes with pi orbitals, Kpp = sqrt(Kpp_i*Kpp_j),
// REQ = (R0, sqrt(E0), Q, Hb).  The numbers are chosen in MMFF/UFF magnitude
// ranges; they are not FireCore's parameter files.
#pragma once
#include <cmath>
#include <cstring>

namespace mmffp {

enum { EL_H = 0, EL_C = 1, EL_N = 2, EL_O = 3, EL_F = 4, EL_S = 5, EL_CL = 6, EL_BR = 7, EL_NA = 8, EL_K = 9, NEL = 10 };

struct Elem {
    const char* sym;
    int valence;       // bonds a neutral atom makes (0: ion / non-bonded only)
    double rcov;       // covalent radius for bond detection [A]
    double R0, E0;     // non-bonded radius [A], well depth [eV]
    double Kss;        // angle stiffness [eV/rad^2]
    double sp3ang;     // rest angle with no pi orbital [deg]
    double Kpp;        // pi-pi stiffness for atoms with pi orbitals [eV]
};

static const Elem kElem[NEL] = {
    {"H", 1, 0.31, 1.50, 0.0020, 0.0, 0.0, 0.0},
    {"C", 4, 0.76, 1.90, 0.0046, 5.0, 109.47, 1.5},
    {"N", 3, 0.71, 1.80, 0.0030, 5.5, 107.0, 1.0},
    {"O", 2, 0.66, 1.75, 0.0026, 6.0, 105.0, 0.5},
    {"F", 1, 0.57, 1.70, 0.0030, 0.0, 0.0, 0.0},
    {"S", 2, 1.05, 2.00, 0.0120, 4.5, 98.0, 0.5},
    {"Cl", 1, 1.02, 2.00, 0.0100, 0.0, 0.0, 0.0},
    {"Br", 1, 1.20, 2.10, 0.0110, 0.0, 0.0, 0.0},
    {"Na", 0, 1.66, 1.60, 0.0040, 0.0, 0.0, 0.0},
    {"K", 0, 2.03, 1.90, 0.0040, 0.0, 0.0, 0.0},
};

inline int elem_index(const char* s) {
    for (int i = 0; i < NEL; i++) if (strcmp(s, kElem[i].sym) == 0) return i;
    return -1;
}

const double kKsp = 1.6;   // pi-sigma stiffness of nodes with pi orbitals [eV]

inline double bond_k(int a, int b) {
    if (a == EL_H || b == EL_H) return 20.0;
    static const double t[4][4] = {{0, 0, 0, 0}, {0, 25.0, 27.0, 28.0}, {0, 27.0, 26.0, 27.5}, {0, 28.0, 27.5, 26.0}};
    if (a < 4 && b < 4) return t[a][b];
    return 20.0;
}
inline double bond_l0(int a, int b) {
    if (a == EL_H || b == EL_H) return 1.09;
    static const double t[4][4] = {{0, 0, 0, 0}, {0, 1.40, 1.38, 1.37}, {0, 1.38, 1.36, 1.35}, {0, 1.37, 1.35, 1.40}};
    if (a < 4 && b < 4) return t[a][b];
    return kElem[a].rcov + kElem[b].rcov;
}

}  // namespace mmffp

// mmff_builder.h -- topology and MMFF parameters from an xyz file and
// FireCore's four parameter tables (ElementTypes / AtomTypes / BondTypes /
// AngleTypes .dat), the work FireCore's drop-in init does through
// MolWorld_sp3::initParams / buildMolecule_xyz / makeFFs
// (cpp/common/molecular/MolWorld_sp3.h:1298-1351, 1359-1586) with
// MMFFparams (MMFFparams.h) and MM::Builder (MMFFBuilder.h).  Host code only.
#pragma once
#include <string>
#include <unordered_map>
#include <vector>

namespace fcb {

// one row of ElementTypes.dat
struct ElementRow {
    std::string name;
    int iZ = 0, neval = 0, valence = 0, piMax = 0;
    double Rcov = 0, RvdW = 0, EvdW = 0;
};

// one row of AtomTypes.dat (angles in degrees as in the file)
struct TypeRow {
    std::string name;
    int iZ = 0, valence = 0, nepair = 0, npi = 0, sym = 0;
    int parent = 0, element = 0, epair = 0;
    double Ruff = 0, RvdW = 0, EvdW = 0, Qbase = 0, Hb = 0;
    double Ass = 0, Asp = 0, Kss = 0, Ksp = 0, Kep = 0, Kpp = 0;
    int sub[3] = {0, 0, 0};   // the X_3 / X_2 / X_1 types of a root type (npi = 0, 1, 2)
};

struct Tables {
    std::vector<ElementRow> elements;
    std::vector<TypeRow> types;
    std::unordered_map<std::string, int> element_index, type_index;
    std::unordered_map<unsigned long long, std::pair<double, double>> bonds;   // (l0, k) by (type, type, order)
    int type(const std::string& s) const {
        auto it = type_index.find(s);
        return it == type_index.end() ? -1 : it->second;
    }
};

// Parses the four tables (DihedralTypes.dat is not needed by this path).
bool load_tables(const char* elem, const char* atom, const char* bond, const char* angle, Tables& T, std::string& err);

// The molecule in MMFFsp3_loc layout: nodes first, then capping atoms, then
// (with electron pairs) the generated pairs; pi orientations after the atoms.
struct Built {
    int natoms = 0, nnode = 0;
    bool pbc = false;                 // the xyz had an "lvs" cell line
    double lvec[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::vector<double> pos;          // (natoms + nnode) x 3
    std::vector<double> REQ;          // natoms x 4
    std::vector<int> type;            // natoms
    std::vector<int> neighs, neighCell;   // natoms x 4 (cells only with pbc)
    std::vector<double> apars, bLs, bKs, Ksp, Kpp;   // nnode x 4
    std::vector<int> permut;          // builder order (xyz atoms read, then electron-pair caps) -> index here
};

// xyz -> Built.  epairs: FireCore's bEpairs (explicit electron pairs and the
// -0.2 e charge moved onto each); nPBC: images searched for the bond cells.
bool build_xyz(const Tables& T, const char* xyz, bool epairs, const int nPBC[3], Built& M, std::string& err);

// REQ of a substrate atom read by name (MMFFparams::loadXYZ semantics):
// (RvdW, sqrt(EvdW), Q, Hb) of the named type, the table's default otherwise.
void substrate_REQ(const Tables& T, const std::string& name, double Q, double H, double REQ[4]);

}  // namespace fcb

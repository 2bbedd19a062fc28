// mmff_host.h -- internal host-side declarations shared by the library's
// translation units (the public C-ABI lives in include/MMFFmulti_lib.h).
#pragma once
#include <cstdint>

// Set the message mmff_last_error() returns (C++ linkage, internal to the library).
void mmff_set_error(const char* msg);
// Add n to the library's kernel-launch count (mmff_kernel_launches).
void mmff_count_launches(int n);

extern "C" {

// Node (heavy atom) count the generator produces for a molecule of natoms atoms.
int mmff_gen_nnode(int natoms);

// Seeded synthetic molecules (C:N:O:H = 10:2:2:10 heavy-atom trees, H caps),
// packed back to back (CSR): per system natoms[s] atoms, nnode = mmff_gen_nnode.
//  topo_mode 0: every system is a replica of one topology (seed);
//            1: system s has its own topology (seed, s).
//  sigma: Gaussian noise per atom coordinate [A]; rotate: random rigid rotation;
//  zplace: z of the lowest atom; cell_xy: molecule centred at cell_xy/2;
//  hbond: assign H-bond pseudo-charges (N/O acceptors -0.7, polar H +0.7);
//  central_cell: PBC image index of the zero shift written into neighCell.
// Returns 0, or -(s+1) if system s could not be generated.
int mmff_gen_systems(int nsys, const int* natoms, uint64_t seed, int topo_mode,
                     double sigma, int rotate, double zplace, const double* cell_xy,
                     int hbond, double* pos, int* neighs, int* neighCell, int* bkneighs,
                     double* REQs, double* apars, double* bLs, double* bKs, double* Ksp,
                     double* Kpp, int* elements, int central_cell);

// Rock-salt (001) slab; returns the number of ions written.
int mmff_gen_slab(double a, int ncell, int layers, double z_top, double q,
                  const double* REQ_cation, const double* REQ_anion,
                  double* spos, double* sREQ);
}

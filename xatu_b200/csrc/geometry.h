// Host-side lattice geometry of the engine (C++), following the semantics of
// Xatu's Lattice class (src/Lattice.cpp).  Row-major arrays, 3 components per
// vector whatever the dimension.
#pragma once
#include <vector>

namespace xatu_geo {

// Lattice::calculateReciprocalLattice (Lattice.cpp:56-80). Returns false if singular.
bool reciprocal_lattice(int ndim, const double* bravais, double* recip);
// Lattice::computeUnitCellArea (Lattice.cpp:119-131).
double unit_cell_area(int ndim, const double* bravais);
// Lattice::generateCombinations (Lattice.cpp:293-312): n^ndim x ndim, dimension 0 fastest.
std::vector<double> combinations(int n, int ndim, bool centered);
// Lattice::brillouinZoneMesh (Lattice.cpp:140-162).
std::vector<double> mp_mesh(int ndim, const double* recip, int n);
// Lattice::reducedBrillouinZoneMesh (Lattice.cpp:172-197): the submesh.
std::vector<double> reduced_mesh(int ndim, const double* recip, int n, int factor);
// Lattice::truncateSupercell / truncateReciprocalSupercell (Lattice.cpp:320-370).
std::vector<double> truncate_supercell(int ndim, const double* basis, int ncell, double radius);
// inv(B B^T) for B = recip (ndim x 3); false if singular.
bool inverse_gram(int ndim, const double* recip, double* inv);
// Lattice::findEquivalentPointBZ (Lattice.cpp:251-279).
int equivalent_point(int ndim, const double* recip, const double* inv, int n_eff, const double* k);
double norm3(const double* v);

}  // namespace xatu_geo

// ctc_wfnfile.h -- contents of a wavefunction file as the library's readers
// leave them (ctc_fchk.cpp for Gaussian formatted checkpoints, ctc_molden.cpp
// for Molden files): the ctc_basis arrays, the atoms and the MO one-particle
// density matrix, all on the host.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

struct ctc_fchk {
  std::string path;
  int32_t natom = 0, nbasis = 0, nalpha = 0, nbeta = 0;
  std::vector<int32_t> numbers;
  std::vector<double> charges, coords;
  // ctc_basis arrays
  std::vector<double> centers, exps, coeffs;
  std::vector<int32_t> shell_atom, nprim, nseg, angmoms;
  std::vector<double> D;  // nbasis x nbasis, row-major (symmetric)
};

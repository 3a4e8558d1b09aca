// mpml.cuh -- M-PML damping ratios of the 3D anisotropic elastic solver (host, mpml.cu).
#pragma once

#include <functional>
#include <vector>

namespace owl {

// u^T B v / u^T v of the damped plane-wave system (mpml_eigenvalue_derivative,
// src/solver/elastic_vhtiort_3d/module_cfspml.f90:51-186) for the orthorhombic
// stiffness c = (c11, c12, c13, c22, c23, c33, c44, c55, c66), damped axis
// (0, 1, 2), ratio and unit wavenumber direction (k1, k2, k3)
double mpml_eig_deriv(const double c[9], int axis, double ratio, double k1, double k2, double k3);
// damp_ratio (module_cfspml.f90:193-248)
float mpml_damp_ratio(const float c[9], int axis);
// cells sampled along a face axis of n cells every `interval` (module_cfspml.f90:290-308)
std::vector<int> mpml_samples(int n, int interval);
// ratio of every cell of an n1 x n2 face (compute_damping_profile_ratio_face,
// module_cfspml.f90:253-409): cell_c(i, j, c) gives the stiffness of face cell
// (i, j); out[j * ld + i]
void mpml_face(int n1, int n2, int axis, const std::function<void(int, int, float*)>& cell_c, float* out, int ld);

}  // namespace owl

// setup_ops.hpp -- host-side set-up of the reference element, the filter and the
// geometry caches of a handle.
#pragma once
#include "../../include/frsdg.h"

#include <utility>
#include <vector>

namespace frsdg
{

struct RefElem
{
    int                 p = 0, n = 0;
    std::vector<double> x, w, D, dL, dR; // D row-major n*n
};

// GLL nodes/weights, differentiation matrix and VCJH correction derivatives.
RefElem build_ref_element(int p, double radau_corr);

// Spectral filter matrix V diag(sigma) V^-1, row-major n*n.
std::vector<double> build_filter_matrix(const RefElem& re, int cut_off, int strength, double alpha);

// Heap-free forms of the two builders above, writing into caller arrays of at
// least n (and n*n for D and F) entries, n = p + 1 <= 10.
void ref_element_into(int p, double radau_corr, double* x, double* w, double* D, double* dL, double* dR);
void filter_matrix_into(int p, const double* x, const double* w, int cut_off, int strength, double alpha,
                        double* F);

struct GeomJacobian
{
    double dx_dcsi, dy_dcsi, dx_deta, dy_deta;
};

// Analytic shape map (csi, eta) in [0,1]^2 -> (x, y), its Jacobian and unit face
// normals: the reference's GeometryModelConc policies (geometry_models.hpp:61-195,
// tests/bump.cpp:13-171, tests/boundary_conforming.cpp:14-120) plus the
// sine-warped periodic map and the Gaussian-bump channel.
class GeometryMap
{
  public:
    explicit GeometryMap(const frsdg_config& c);
    std::pair<double, double> physical(double csi, double eta) const;
    GeomJacobian              jacobian(double csi, double eta) const;
    std::pair<double, double> x_face_normal(double csi, double eta) const;
    std::pair<double, double> y_face_normal(double csi, double eta) const;
    // constant diagonal metrics (no per-node cache needed)
    bool affine() const;

  private:
    std::pair<double, double> wall(double x) const; // (h, dh/dx)
    int    kind_, profile_;
    double Lx_, Ly_, prm_[4];
};

} // namespace frsdg

// q2d_setup.h — host-side geometry setup of one block (Setup_Metrics, Mod_Metrics.f90:11-148).
// Setup runs once per block on the host, in IEEE double arithmetic without FMA contraction,
// and produces the SoA planes the device kernels read.
#pragma once
#include <vector>
#include "../../include/q2d_gpu.h"

namespace q2d {

struct HostGeom {
    int ni = 0, nj = 0;
    // ghost-frame arrays (i, j in [-2, n+1], 0-based): index (j+2)*(ni+4) + (i+2)
    std::vector<double> M;     // 4 per cell: M11 M12 M21 M22
    std::vector<double> dl;    // 2 per cell
    std::vector<double> sur;   // 1 per cell
    std::vector<double> fi;    // (ni+1)*nj i-faces x (nx, ny, len), face F of row j at j*(ni+1)+F
    std::vector<double> fj;    // ni*(nj+1) j-faces x (nx, ny, len), face G of column i at G*ni+i
    std::vector<double> src0, src1;   // interior: 1/r (axi) or Gx, Gy (area)
    int g(int i, int j) const { return (j + 2) * (ni + 4) + (i + 2); }
};

// Interior metrics, face normals and source geometry of a block. nodes: (2, 0:ni, 0:nj)
// Fortran order; area: nodal cross-section or nullptr. Returns a Q2D_* status.
int setup_block(int ni, int nj, const double* nodes, const double* area, int source, HostGeom& G);

// Ghost-cell metrics of one boundary record (BC_Connect_Metrics / BC_Symmetry_Metrics /
// BC_Extrapolate_Metrics, Lib_Metrics.f90:285-553). donor/donor_nodes only for type 101.
int ghost_metrics(const q2d_bc_rec& r, int ni, int nj, const double* nodes, HostGeom& G,
                  int dni, int dnj, const double* donor_nodes);

// Unit tangent of the boundary face of a record (Setup_Inflow_Geometry, Lib_BC_Fluxes_Inflow.f90:521-531).
void face_tangent(const q2d_bc_rec& r, int ni, const double* nodes, double* t0, double* t1);

// versor(d,:) = M(d,:)/norm2(M(d,:)) of an interior cell (Mod_dt.f90:83).
void versors(const HostGeom& G, int i, int j, double* v);

}  // namespace q2d

/*
 * monitors.cpp -- surface integrals of a boundary zone (TEST INFRASTRUCTURE).
 *
 * Restates the integrals the reference's surface monitors are built from,
 * Mesh/QuadMesh_Integrals.incf:
 *   Compute_ScalarScalarSurfaceIntegral  :67-166   "Surface", "pressure"
 *   Compute_ScalarVectorSurfaceIntegral  :168-206  "pressure" (force)
 *   Compute_VectorVectorSurfaceIntegral  :208-284  "mass-flow", "flow"
 *   Compute_TensorVectorSurfaceIntegral  :286-346  "viscous", with ComputeViscousTensor
 *                                                  (Physics/ViscousFluxes.f90:416-461)
 * over the boundary edges' storage(1) traces (Q and dQ) as they stand, i.e. those of the last
 * residual evaluation -- after a time step, the last stage's input state, as the reference's
 * monitors (updated after TimeStep, DGTimeIntegrator.f90:194-208) read them.  Straight edges use
 * n(:,0) and dS(0) at every node, curved edges the per-node values; the pressure is getPressure1D
 * (Physics/VariableConversion.f90:56-71).  Values are dimensionless, as the mesh functions return
 * them; the monitors' reference-value factors (Monitors.f90:1109-1141) are applied by the caller.
 */
#include "oracle_internal.h"
#include <cmath>

namespace orc {

void surface_integrals(const Oracle& o, int zone, double out[8]) {
  for (int k = 0; k < 8; ++k) out[k] = 0.0;
  const Physics& ph = o.ph;
  const double mu = ph.mu, lambda = ph.lambda, gm1 = ph.gm1;
  double surf = 0.0, pint = 0.0, fpx = 0.0, fpy = 0.0, vx = 0.0, vy = 0.0, mflow = 0.0, flow = 0.0;
  for (int id : o.zones[zone].edges) {
    const Edge& f = o.ed[id];
    const EdgeStorage& st = f.storage[0];
    const int P = f.P();
    const std::vector<double>& w = f.sp->w;
    const bool curved = f.is_curved();
    // the scalar integrals form per-edge sums first (sum / dot_product), as the reference does
    double s_surf = 0.0, s_p = 0.0;
    for (int j = 0; j < P; ++j) {
      const double* Q = &st.Q[4 * j];
      const double dS = curved ? f.dS[j] : f.dS[0];
      const double p = gm1 * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]);
      s_surf = s_surf + w[j] * dS;
      s_p = s_p + p * dS * w[j];
    }
    surf = surf + s_surf;
    pint = pint + s_p;
    for (int j = 0; j < P; ++j) {
      const double* Q = &st.Q[4 * j];
      const double dS = curved ? f.dS[j] : f.dS[0];
      const double nx = f.nx(j), ny = f.ny(j);
      const double p = gm1 * (Q[3] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2]) / Q[0]);
      fpx = fpx + p * w[j] * nx * dS;
      fpy = fpy + p * w[j] * ny * dS;
      mflow = mflow + w[j] * (Q[1] * nx + Q[2] * ny) * dS;
      flow = flow + w[j] * (Q[1] * nx + Q[2] * ny) * dS / Q[0];
      if (o.cas.navier_stokes && !st.dQ.empty()) {
        const double* gx = &st.dQ[(0 * P + j) * 4];
        const double* gy = &st.dQ[(1 * P + j) * 4];
        const double invRho = 1.0 / Q[0];
        const double u = Q[1] * invRho, v = Q[2] * invRho;
        const double uDivRho = u * invRho, vDivRho = v * invRho;
        const double divV = -uDivRho * gx[0] + invRho * gx[1] - vDivRho * gy[0] + invRho * gy[2];
        const double txx = 2.0 * mu * (-uDivRho * gx[0] + invRho * gx[1]) + lambda * mu * divV;
        const double tyy = 2.0 * mu * (-vDivRho * gy[0] + invRho * gy[2]) + lambda * mu * divV;
        const double txy = -mu * vDivRho * gx[0] - mu * uDivRho * gy[0] + mu * invRho * gy[1] + mu * invRho * gx[2];
        vx = vx + w[j] * (txx * nx + txy * ny) * dS;
        vy = vy + w[j] * (txy * nx + tyy * ny) * dS;
      }
    }
  }
  out[0] = surf; out[1] = pint; out[2] = fpx; out[3] = fpy; out[4] = vx; out[5] = vy; out[6] = mflow; out[7] = flow;
}

}  // namespace orc

extern "C" int or_probe(void* h, int e, double xi, double eta, double out[4]) {
  // Probe_t update (Monitors.f90:740-830): BilinearForm(Q, l_xi, l_eta) = dot_product(l_xi, Q l_eta)
  // (Generic/MatrixOperations.f90:185-209), with the element's Lagrange basis at (xi, eta)
  orc::Oracle& o = *static_cast<orc::Oracle*>(h);
  if (e < 0 || e >= int(o.el.size())) return -1;
  const orc::Element& E = o.el[e];
  const int P = E.P;
  const std::vector<double> lx = E.sp->lj(xi), ly = E.sp->lj(eta);
  const double* Q = &o.Q[E.offset];
  for (int v = 0; v < 4; ++v) {
    double b = 0.0;
    for (int i = 0; i < P; ++i) {
      double t = 0.0;
      for (int j = 0; j < P; ++j) t += Q[(j * P + i) * 4 + v] * ly[j];
      b += lx[i] * t;
    }
    out[v] = b;
  }
  return 0;
}

extern "C" int or_surface_integrals(void* h, int zone, double out[8]) {
  orc::Oracle& o = *static_cast<orc::Oracle*>(h);
  if (zone < 1 || zone >= int(o.zones.size())) return -1;
  orc::surface_integrals(o, zone, out);
  return 0;
}

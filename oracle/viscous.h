/*
 * viscous.h -- Navier-Stokes terms of the oracle (TEST INFRASTRUCTURE).
 * See viscous.cpp for the reference routines each function restates.
 */
#pragma once
#include "oracle_internal.h"

namespace orc {

struct ViscousWork {
  int dummy = 0;
};

void riemann(const Physics& ph, int which, const double* qL, const double* qR, double nx, double ny, double* F);
void inviscid_flux(const Physics& ph, const double* u, double* f, double* g);
double pressure(const Physics& ph, const double* Q);

void viscous_wall_associate(Oracle& o, Zone& Z, Edge& f);
void viscous_wall_update(Oracle& o, Zone& Z, Edge& f);
void dirichlet_viscous_update(Oracle& o, Zone& Z, Edge& f);
void farfield_update(Oracle& o, Zone& Z, Edge& f);
void pressure_outlet_update(Oracle& o, Zone& Z, Edge& f);

void compute_gradient(Oracle& o, ViscousWork& vw);
void viscous_volume_flux(Oracle& o, Element& e, std::vector<double>& F, ViscousWork& vw);
void viscous_interior_flux(Oracle& o, Edge& f, const std::vector<double>& QL, const std::vector<double>& QR,
                           std::vector<double>& Fs, ViscousWork& vw);
void viscous_interior_gradient_faces(Oracle& o, Edge& f, const std::vector<double>& QL, const std::vector<double>& QR,
                                     ViscousWork& vw);
void viscous_mortar_fluxes(Oracle& o, Edge& f, const std::vector<double>& QLN, const std::vector<double>& QRN,
                           const std::vector<double>& QLS, const std::vector<double>& QRS,
                           std::vector<double>& FN, std::vector<double>& FS, ViscousWork& vw);
void viscous_mortar_gradient_faces(Oracle& o, Edge& f, const std::vector<double>& QLN, const std::vector<double>& QRN,
                                   const std::vector<double>& QLS, const std::vector<double>& QRS, ViscousWork& vw);
void viscous_boundary_flux(Oracle& o, Edge& f, std::vector<double>& F, ViscousWork& vw);
void viscous_boundary_gradient_face(Oracle& o, Edge& f, ViscousWork& vw);
void interior_gradient(Oracle& o, Element& e, double* dQ);   // dQ[(d*NP+q)*4+k]

// dissipation.cpp
double edge_jumps(const Oracle& o, const Edge& f, int var);
double av_element_viscosity(const Oracle& o, const Element& e);
double av_edge_viscosity(const Oracle& o, const Edge& f);
void compute_av_viscosity(Oracle& o);
void set_physical_av(Oracle& o);
bool laplacian_av(const Oracle& o);
void av_volume_flux(Oracle& o, Element& e, std::vector<double>& F);
void av_face_flux(const Oracle& o, const Edge& f, const double* qL, const double* qR, double* Fa);

}  // namespace orc

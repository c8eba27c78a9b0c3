/*
 * viscous.cpp -- Navier-Stokes terms of the oracle (TEST INFRASTRUCTURE).
 *
 * Placeholder bodies: the oracle currently restates the Euler build
 * (Makefile target Euler, no -DNAVIER_STOKES).  Calls with navier_stokes != 0
 * raise.
 */
#include "viscous.h"
#include <stdexcept>

namespace orc {

[[noreturn]] static void ns_missing() { throw std::runtime_error("Navier-Stokes terms are not available in the oracle"); }

void viscous_wall_associate(Oracle&, Zone&, Edge&) { ns_missing(); }
void viscous_wall_update(Oracle&, Zone&, Edge&) { ns_missing(); }
void dirichlet_viscous_update(Oracle&, Zone&, Edge&) { ns_missing(); }
void farfield_update(Oracle&, Zone&, Edge&) { ns_missing(); }
void pressure_outlet_update(Oracle&, Zone&, Edge&) { ns_missing(); }
void compute_gradient(Oracle&, ViscousWork&) { ns_missing(); }
void viscous_volume_flux(Oracle&, Element&, std::vector<double>&, ViscousWork&) { ns_missing(); }
void viscous_interior_flux(Oracle&, Edge&, const std::vector<double>&, const std::vector<double>&, std::vector<double>&,
                           ViscousWork&) { ns_missing(); }
void viscous_interior_gradient_faces(Oracle&, Edge&, const std::vector<double>&, const std::vector<double>&, ViscousWork&) {
  ns_missing();
}
void viscous_mortar_fluxes(Oracle&, Edge&, const std::vector<double>&, const std::vector<double>&, const std::vector<double>&,
                           const std::vector<double>&, std::vector<double>&, std::vector<double>&, ViscousWork&) {
  ns_missing();
}
void viscous_mortar_gradient_faces(Oracle&, Edge&, const std::vector<double>&, const std::vector<double>&,
                                   const std::vector<double>&, const std::vector<double>&, ViscousWork&) {
  ns_missing();
}
void viscous_boundary_flux(Oracle&, Edge&, std::vector<double>&, ViscousWork&) { ns_missing(); }
void viscous_boundary_gradient_face(Oracle&, Edge&, ViscousWork&) { ns_missing(); }

}  // namespace orc

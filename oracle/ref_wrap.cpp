// C entry points over the reference's own LPS and bond-based kernels, compiled
// from the reference sources (src/materials/elastic.cxx,
// src/materials/elastic_bond_based.cxx, src/materials/material_utilities.cxx,
// src/core/Peridigm_InfluenceFunction.cpp, src/io/discretization/Peridigm_GeometryUtils.cpp)
// by oracle/Makefile into oracle/_ref/.
// Test infrastructure only: the product never links this library.
#include <stdexcept>
#include <string>
#include "material_utilities.h"
#include "elastic.h"
#include "elastic_bond_based.h"
#include "Peridigm_GeometryUtils.hpp"

extern "C" {

// PeridigmNS::InfluenceFunction::setInfluenceFunction (src/core/Peridigm_InfluenceFunction.hpp:121).
// Returns 0 on success, 1 when the reference rejects the name.
int pdref_set_influence(const char* name) {
  try {
    PeridigmNS::InfluenceFunction::self().setInfluenceFunction(std::string(name));
  } catch (const std::exception&) {
    return 1;
  }
  return 0;
}

// MATERIAL_EVALUATION::computeWeightedVolume (src/materials/material_utilities.cxx:501-520).
void pdref_weighted_volume(const double* x, const double* vol, double* m, int n_owned,
                           const int* nl, double horizon) {
  MATERIAL_EVALUATION::computeWeightedVolume(x, vol, m, n_owned, nl, horizon);
}

// MATERIAL_EVALUATION::computeDilatation<double> (src/materials/material_utilities.cxx:235-289).
void pdref_dilatation(const double* x, const double* y, const double* m, const double* vol,
                      const double* bond_damage, double* theta, const int* nl, int n_owned,
                      double horizon) {
  MATERIAL_EVALUATION::computeDilatation<double>(x, y, m, vol, bond_damage, theta, nl, n_owned,
                                                 horizon);
}

// MATERIAL_EVALUATION::computeInternalForceLinearElastic<double> (src/materials/elastic.cxx:55-146).
// The caller zeroes f first, as ElasticMaterial::computeForce does
// (src/materials/Peridigm_ElasticMaterial.cpp:149).
void pdref_force_linear_elastic(const double* x, const double* y, const double* m,
                                const double* vol, const double* theta,
                                const double* bond_damage, double* f, const int* nl, int n_owned,
                                double K, double mu, double horizon) {
  MATERIAL_EVALUATION::computeInternalForceLinearElastic<double>(
      x, y, m, vol, theta, bond_damage, f, nullptr, nl, n_owned, K, mu, horizon, 0.0, nullptr);
}

// MATERIAL_EVALUATION::computeInternalForceElasticBondBased<double>
// (src/materials/elastic_bond_based.cxx:55-124); the caller zeroes f first, as
// ElasticBondBasedMaterial::computeForce does (Peridigm_ElasticBondBasedMaterial.cpp:116).
void pdref_force_bond_based(const double* x, const double* y, const double* vol, const double* bond_damage,
                            double* f, const int* nl, int n_owned, double K, double horizon, int plane,
                            double height) {
  MATERIAL_EVALUATION::computeInternalForceElasticBondBased<double>(x, y, vol, bond_damage, f, nl, n_owned, K,
                                                                    horizon, plane != 0, height);
}

// PeridigmNS::hexCentroidAndVolume / tetCentroidAndVolume
// (src/io/discretization/Peridigm_GeometryUtils.cpp:52-339): the point an
// Exodus element becomes (nodes: 8 or 4 xyz triples).
void pdref_hex_centroid_volume(double* nodes, double* centroid, double* volume) {
  PeridigmNS::hexCentroidAndVolume(nodes, centroid, volume);
}
void pdref_tet_centroid_volume(double* nodes, double* centroid, double* volume) {
  PeridigmNS::tetCentroidAndVolume(nodes, centroid, volume);
}

}  // extern "C"

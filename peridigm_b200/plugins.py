"""Host-side mirror of Peridigm's plugin interfaces for the hot path.

Names, arguments and field names follow the reference so a caller (or a test)
reads like Peridigm code:

* ``ElasticMaterial``            PeridigmNS::ElasticMaterial (src/materials/Peridigm_ElasticMaterial.{hpp,cpp})
* ``CriticalStretchDamageModel`` PeridigmNS::CriticalStretchDamageModel (src/damage/Peridigm_CriticalStretchDamageModel.cpp)
* ``ModelEvaluator``             PeridigmNS::ModelEvaluator::evalModel (src/core/Peridigm_ModelEvaluator.cpp:57-131)
* ``DataManager``                the NONE/N/NP1 fields the plugins read and write (src/core/Peridigm_DataManager.hpp)

All arithmetic runs in the CUDA library; these classes only move arrays.
"""
from __future__ import annotations

import numpy as np

from .context import Context


def calculate_bulk_modulus(params):
    """Material::calculateBulkModulus (src/materials/Peridigm_Material.cpp:335-384)."""
    p = params
    if "Bulk Modulus" in p:
        return float(p["Bulk Modulus"])
    if "Shear Modulus" in p and "Young's Modulus" in p:
        E, mu = float(p["Young's Modulus"]), float(p["Shear Modulus"])
        return E * mu / (3.0 * (3.0 * mu - E))
    if "Shear Modulus" in p and "Poisson's Ratio" in p:
        mu, nu = float(p["Shear Modulus"]), float(p["Poisson's Ratio"])
        return 2.0 * mu * (1.0 + nu) / (3.0 * (1.0 - 2.0 * nu))
    if "Young's Modulus" in p and "Poisson's Ratio" in p:
        E, nu = float(p["Young's Modulus"]), float(p["Poisson's Ratio"])
        return E / (3.0 * (1.0 - 2.0 * nu))
    raise ValueError("**** Error:  Exactly two elastic constants must be provided.")


def calculate_shear_modulus(params):
    """Material::calculateShearModulus (src/materials/Peridigm_Material.cpp:386-433)."""
    p = params
    if "Shear Modulus" in p:
        return float(p["Shear Modulus"])
    if "Bulk Modulus" in p and "Young's Modulus" in p:
        K, E = float(p["Bulk Modulus"]), float(p["Young's Modulus"])
        return 3.0 * K * E / (9.0 * K - E)
    if "Bulk Modulus" in p and "Poisson's Ratio" in p:
        K, nu = float(p["Bulk Modulus"]), float(p["Poisson's Ratio"])
        return 3.0 * K * (1.0 - 2.0 * nu) / (2.0 * (1.0 + nu))
    if "Young's Modulus" in p and "Poisson's Ratio" in p:
        E, nu = float(p["Young's Modulus"]), float(p["Poisson's Ratio"])
        return E / (2.0 * (1.0 + nu))
    raise ValueError("**** Error:  Exactly two elastic constants must be provided.")


class DataManager:
    """Fields of one block in a single-process run (owned points only).

    getData(name, step) returns the numpy array of a field; step is
    "NONE", "N" or "NP1" as in PeridigmField::Step. updateState copies NP1 to N
    (DataManager::updateState, Peridigm_DataManager.hpp:159).
    """

    TWO_STEP = ("Coordinates", "Dilatation", "Bond_Damage", "Force_Density", "Damage", "Displacement", "Velocity")

    def __init__(self, num_points, num_bonds):
        self.n = int(num_points)
        self.nb = int(num_bonds)
        self.fields = {}
        for name, size in [("Model_Coordinates", 3), ("Volume", 1), ("Weighted_Volume", 1)]:
            self.fields[(name, "NONE")] = np.zeros(size * self.n)
        for name, size in [("Coordinates", 3), ("Dilatation", 1), ("Force_Density", 3), ("Damage", 1),
                           ("Displacement", 3), ("Velocity", 3)]:
            for st in ("N", "NP1"):
                self.fields[(name, st)] = np.zeros(size * self.n)
        for st in ("N", "NP1"):
            self.fields[("Bond_Damage", st)] = np.zeros(self.nb)

    def getData(self, name, step="NONE"):
        if name not in self.TWO_STEP:
            step = "NONE"
        return self.fields[(name, step)]

    def updateState(self):
        for name in self.TWO_STEP:
            self.fields[(name, "N")][:] = self.fields[(name, "NP1")]


def _neighbor_list_count(nl, n):
    k, nb = 0, 0
    for _ in range(n):
        c = int(nl[k])
        nb += c
        k += c + 1
    return nb


class _Bound:
    """Lazily creates the device context the first time a data manager is seen."""

    def __init__(self, precision, influence):
        self.precision = precision
        self.influence = influence
        self.ctx = None
        self.key = None

    def context(self, neighborhoodList, dataManager, horizon, configure):
        key = (id(dataManager), id(neighborhoodList))
        if self.ctx is None or self.key != key:
            ctx = Context(precision=self.precision, influence=self.influence)
            ctx.set_points(dataManager.getData("Model_Coordinates"), dataManager.getData("Volume"))
            ctx.set_horizons([horizon])
            ctx.set_bonds(neighborhoodList)
            configure(ctx)
            self.ctx, self.key = ctx, key
        return self.ctx


class ElasticMaterial:
    """PeridigmNS::ElasticMaterial: LPS "Elastic" material.

    Parameters as in the reference ParameterList: "Density", two elastic
    constants ("Bulk Modulus", "Shear Modulus", ...), "Horizon".
    """

    def __init__(self, params, precision="fp64", influence="One"):
        self.m_bulkModulus = calculate_bulk_modulus(params)
        self.m_shearModulus = calculate_shear_modulus(params)
        self.m_density = float(params["Density"])
        self.m_horizon = float(params["Horizon"])
        self._b = _Bound(precision, influence)

    def Name(self):
        return "Elastic"

    def Density(self):
        return self.m_density

    def BulkModulus(self):
        return self.m_bulkModulus

    def ShearModulus(self):
        return self.m_shearModulus

    def _ctx(self, nl, dm):
        return self._b.context(nl, dm, self.m_horizon,
                               lambda c: c.material(self.m_bulkModulus, self.m_shearModulus, self.m_density))

    def initialize(self, dt, numOwnedPoints, ownedIDs, neighborhoodList, dataManager):
        """ElasticMaterial::initialize (Peridigm_ElasticMaterial.cpp:124-139)."""
        ctx = self._ctx(neighborhoodList, dataManager)
        dataManager.getData("Weighted_Volume")[:] = ctx.weighted_volume()

    def computeForce(self, dt, numOwnedPoints, ownedIDs, neighborhoodList, dataManager):
        """ElasticMaterial::computeForce (Peridigm_ElasticMaterial.cpp:141-172): zero the
        force, computeDilatation, computeInternalForceLinearElastic, on the NP1 bond damage."""
        ctx = self._ctx(neighborhoodList, dataManager)
        ctx.set_bond_damage(dataManager.getData("Bond_Damage", "NP1"))
        f = ctx.compute_force(dataManager.getData("Coordinates", "NP1"))
        dataManager.getData("Force_Density", "NP1")[:] = f
        dataManager.getData("Dilatation", "NP1")[:] = ctx.field("Dilatation")


class CriticalStretchDamageModel:
    """PeridigmNS::CriticalStretchDamageModel ("Critical Stretch")."""

    def __init__(self, params, precision="fp64"):
        self.m_criticalStretch = float(params["Critical Stretch"])
        if "Thermal Expansion Coefficient" in params:
            raise NotImplementedError("thermal strains are outside this build's hot path")
        self._b = _Bound(precision, "One")
        self.horizon = float(params.get("Horizon", 1.0))

    def Name(self):
        return "Critical Stretch"

    def _ctx(self, nl, dm):
        def configure(c):
            c.material(1.0, 1.0, 1.0)  # the damage law reads no material constant
            c.critical_stretch(self.m_criticalStretch)
        return self._b.context(nl, dm, self.horizon, configure)

    def initialize(self, dt, numOwnedPoints, ownedIDs, neighborhoodList, dataManager):
        """Zero node and bond damage (Peridigm_CriticalStretchDamageModel.cpp:83-106)."""
        dataManager.getData("Damage", "NP1")[:] = 0.0
        dataManager.getData("Bond_Damage", "NP1")[:] = 0.0

    def computeDamage(self, dt, numOwnedPoints, ownedIDs, neighborhoodList, dataManager):
        """CriticalStretchDamageModel::computeDamage (Peridigm_CriticalStretchDamageModel.cpp:108-184)."""
        ctx = self._ctx(neighborhoodList, dataManager)
        ctx.set_bond_damage(dataManager.getData("Bond_Damage", "N"))
        ctx.compute_damage(dataManager.getData("Coordinates", "NP1"))
        dataManager.getData("Bond_Damage", "NP1")[:] = ctx.field("Bond_Damage")
        dataManager.getData("Damage", "NP1")[:] = ctx.field("Damage")


class ModelEvaluator:
    """ModelEvaluator::evalModel (Peridigm_ModelEvaluator.cpp:57-131) for one block,
    fused on the device: damage -> dilatation -> force in two bond passes."""

    def __init__(self, material, damage=None, precision="split", influence="One"):
        self.material = material
        self.damage = damage
        self._b = _Bound(precision, influence)

    def _ctx(self, nl, dm):
        def configure(c):
            c.material(self.material.BulkModulus(), self.material.ShearModulus(), self.material.Density())
            if self.damage is not None:
                c.critical_stretch(self.damage.m_criticalStretch)
        return self._b.context(nl, dm, self.material.m_horizon, configure)

    def evalModel(self, neighborhoodList, dataManager):
        ctx = self._ctx(neighborhoodList, dataManager)
        ctx.set_bond_damage(dataManager.getData("Bond_Damage", "N"))
        f = ctx.compute_force(dataManager.getData("Coordinates", "NP1"))
        dataManager.getData("Force_Density", "NP1")[:] = f
        dataManager.getData("Dilatation", "NP1")[:] = ctx.field("Dilatation")
        dataManager.getData("Bond_Damage", "NP1")[:] = ctx.field("Bond_Damage")
        dataManager.getData("Damage", "NP1")[:] = ctx.field("Damage")
        if not dataManager.getData("Weighted_Volume").any():
            dataManager.getData("Weighted_Volume")[:] = ctx.weighted_volume()

"""CPU slab engine over the oracle, for the multi-rank tests (test
infrastructure: the oracle is the checker, never the product).

Velocity-Verlet in the order of Peridigm::executeExplicit
(src/core/Peridigm.cpp:1447-1590), structured like the library's stepping
form: begin (initial evaluation, first half of step 1), step, finish; pack and
unpack move (u, y) of listed local points.
"""
import numpy as np

from oracle import oracle as O


class OracleEngine:
    def __init__(self, w):
        self.x = np.asarray(w["x"], dtype=np.float64)
        self.vol = np.asarray(w["vol"], dtype=np.float64)
        n = len(self.vol)
        self.h = float(w["horizon"])
        self.row, self.col = O.neighbor_search(self.x, self.h, w.get("planes"))
        self.m = O.weighted_volume(self.x, self.vol, self.row, self.col, self.h)
        self.K, self.mu, self.rho, self.s_c = w["K"], w["mu"], float(w["rho"]), w.get("s_c")
        self.u = np.zeros(3 * n)
        self.v = np.asarray(w["v0"], dtype=np.float64).copy()
        self.dmg = np.zeros(len(self.col))
        self.mask = np.zeros(3 * n, dtype=bool)
        self.bc_a = np.zeros(3 * n)
        self.bc_b = np.zeros(3 * n)
        for bc in w.get("bcs", []):
            k = 3 * np.asarray(bc["points"], dtype=np.int64) + bc["coordinate"]
            self.mask[k] = True
            self.bc_a[k] = bc["a"]
            self.bc_b[k] = bc["b"]

    def _eval(self, commit):
        y = self.x + self.u
        r = O.eval_model(self.x, y, self.vol, self.row, self.col, self.K, self.mu, self.h, s_c=self.s_c,
                         dmg_n=self.dmg, m=self.m)
        if commit:
            self.dmg = r["bond_damage"]
        return r["force"] / self.rho

    def _advance(self, acc, step, last):
        dt = self.dt
        if step > 0:
            self.v = self.v + (dt / 2.0) * acc  # end of step `step` (Peridigm.cpp:1577)
        if last:
            return
        vh = self.v + (dt / 2.0) * acc  # first half of the next step (:1480)
        tc, tp = self.t0 + (step + 1) * dt, self.t0 + step * dt
        d = (self.bc_a * tc + self.bc_b) - (self.bc_a * tp + self.bc_b)
        vh[self.mask] = d[self.mask] / (tc - tp)  # DirichletIncrementBC (Peridigm_BoundaryCondition.cpp:235)
        self.v = vh
        self.u = self.u + dt * vh  # (:1501)

    def begin(self, dt, t0):
        self.dt, self.t0, self.s = float(dt), float(t0), 0
        self._advance(self._eval(False), 0, False)

    def step(self, k):
        for _ in range(k):
            self.s += 1
            self._advance(self._eval(True), self.s, False)

    def finish(self):
        self.s += 1
        self._advance(self._eval(True), self.s, True)
        return {"steps": self.s}

    def pack(self, idx, out):
        i = idx.numpy().astype(np.int64)
        u3 = self.u.reshape(-1, 3)
        out[:, :3] = __import__("torch").from_numpy(u3[i])
        out[:, 3:] = __import__("torch").from_numpy(self.x.reshape(-1, 3)[i] + u3[i])

    def unpack(self, idx, vals):
        i = idx.numpy().astype(np.int64)
        self.u.reshape(-1, 3)[i] = vals[:, :3].numpy()

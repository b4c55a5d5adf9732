"""Generates the golden fixtures of the large-workload parity tests with the
oracle (the FP64 C++ restatement of the reference CPU MPS path).

The oracle needs minutes for these workloads, longer than a GPU test should
wait, so its results are committed here and the GPU tests compare against
them.  Each fixture stores the workload's generator arguments next to the
results, and the tests rebuild the circuit from those.

  python tests/golden/make_fixtures.py [config1_exact] [config1_drift] [config3_hea] [config4_prefix]

* config1_exact.npz: the 50-qubit, depth-40, chi 128 random circuit under the
  exact split rule (every split an exact SVD): <0...0|psi> and every split
  record (site, shape, path, kept chi, discarded weight).
* config1_drift.npz: the oracle against itself on that workload, Golub-Kahan
  against its Jacobi as the primary SVD: per-split discarded-weight drift
  and the drift of the norm and of normalised <Z_q>.
* config3_hea.npz: the 32-qubit, 8-layer hardware-efficient ansatz at chi 64:
  the observable sum Z_i Z_i+1 + 0.5 sum X_i and its parameter-shift
  derivative for 16 of the 512 parameters (two oracle runs each).
* config4_prefix.npz: the first layers of the 100-qubit chi 256 block
  circuit under the exact split rule: amplitude and split records.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "wqc-core_b200"))

import oracle as O  # noqa: E402
from wqc_cuda import circuits as C  # noqa: E402

CONFIG4_PREFIX_LAYERS = 12
CONFIG3_PARAMS = np.arange(0, 512, 32) + np.arange(16) % 7  # 16 parameters spread over the layers


def config1_exact():
    w = C.config1()
    t0 = time.time()
    o = O.run(w.n, w.chi, w.gates, rule=1)
    rec = o.records()
    z_sites = np.array([0, 12, 25, 37, 49])
    z = [o.expectation(["".join("Z" if w.n - 1 - i == q else "I" for i in range(w.n))], [1.0]).real for q in z_sites]
    np.savez_compressed(os.path.join(HERE, "config1_exact.npz"), n=w.n, depth=40, chi=w.chi, seed=w.seed,
                        amplitude=np.array(o.amplitude_zero()), records=rec, bond_dims=o.bond_dims(),
                        norm2=o.expectation(["I" * w.n], [1.0]).real, z_sites=z_sites, z=np.array(z))
    print(f"config1_exact: {len(rec)} splits, amplitude {o.amplitude_zero()}, {time.time() - t0:.0f} s")


def config1_drift():
    """The oracle against itself on the config1_exact workload: Golub-Kahan
    (nalgebra's family, the reference's primary SVD) and the one-sided
    Jacobi of svd_guard.rs as primary SVD.  Both are FP64 SVDs of the same
    matrices; their per-split discarded weights and final state drift apart
    as truncation carries rounding differences on.  That drift bounds what
    agreement with any other FP64 SVD (the device's Jacobi) can mean."""
    w = C.config1()
    z_sites = np.array([0, 12, 25, 37, 49])
    runs = []
    for primary in (0, 1):
        O.set_primary_svd(primary)
        t0 = time.time()
        o = O.run(w.n, w.chi, w.gates, rule=1)
        norm2 = o.expectation(["I" * w.n], [1.0]).real
        z = [o.expectation(["".join("Z" if w.n - 1 - i == q else "I" for i in range(w.n))], [1.0]).real / norm2
             for q in z_sites]
        runs.append((o.records(), norm2, np.array(z)))
        print(f"config1_drift: primary SVD {primary} in {time.time() - t0:.0f} s, norm2 {norm2}")
    O.set_primary_svd(0)
    (r0, n0, z0), (r1, n1, z1) = runs
    assert all(np.array_equal(r0[k], r1[k]) for k in ("left_site", "rows", "cols", "path", "chi"))
    np.savez_compressed(os.path.join(HERE, "config1_drift.npz"),
                        weight_drift=np.abs(r0["discarded_weight"] - r1["discarded_weight"]),
                        norm2_rel_drift=abs(n0 - n1) / abs(n0), z_norm_drift=np.abs(z0 - z1).max())


def config3_hea():
    n, layers, chi = 32, 8, 64
    gates, pidx, params = C.hea_ansatz(n, layers)
    labels, coeffs = C.zz_x_observable(n)
    t0 = time.time()
    o = O.run(n, chi, gates)
    value = o.expectation(labels, coeffs).real
    grads = []
    for p in CONFIG3_PARAMS:
        inst = np.nonzero(pidx == p)[0]
        assert len(inst) == 1
        vals = []
        for sgn in (1.0, -1.0):
            g = gates.copy()
            g["angle"][inst[0]] += sgn * np.pi / 2
            vals.append(O.run(n, chi, g).expectation(labels, coeffs).real)
        grads.append(0.5 * (vals[0] - vals[1]))
    np.savez_compressed(os.path.join(HERE, "config3_hea.npz"), n=n, layers=layers, chi=chi, value=value,
                        params=CONFIG3_PARAMS, shift_grad=np.array(grads), records=o.records())
    print(f"config3_hea: value {value}, {len(grads)} shift derivatives, {time.time() - t0:.0f} s")


def config4_prefix():
    w = C.config4(CONFIG4_PREFIX_LAYERS)
    t0 = time.time()
    o = O.run(w.n, w.chi, w.gates, rule=1)
    rec = o.records()
    np.savez_compressed(os.path.join(HERE, "config4_prefix.npz"), layers=CONFIG4_PREFIX_LAYERS, chi=w.chi,
                        seed=w.seed, amplitude=np.array(o.amplitude_zero()), records=rec, bond_dims=o.bond_dims())
    print(f"config4_prefix: {len(rec)} splits ({int(np.sum(rec['rows'] == 512))} at 512 x 512), "
          f"amplitude {o.amplitude_zero()}, {time.time() - t0:.0f} s")


if __name__ == "__main__":
    todo = sys.argv[1:] or ["config1_exact", "config1_drift", "config3_hea", "config4_prefix"]
    for name in todo:
        globals()[name]()

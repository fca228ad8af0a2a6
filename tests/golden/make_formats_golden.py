"""Write the reference's on-disk table formats with the reference's own writers.

    LIGHTHIT_REFERENCE_SRC=<reference src> LIGHTHIT_FIXTURE_WORK=<scratch> \\
        python tests/golden/make_formats_golden.py

Slices of the committed tables (a few intervals and frequencies, so the files
stay small) are written by ``band_fold.save_folded`` (``folded.npy`` +
``folded.json``), ``Ge2KernelStore.save`` (``pack.json`` + ``<n>.npy``) and
``ResponseCache.save`` (``transport-450.npz``) into ``tests/golden/formats/``;
``tests/test_formats.py`` rebuilds the same slices (and seeded coefficients)
and checks ``lighthit_b200.formats`` against the files the reference wrote.
"""
import shutil
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(Path(__file__).resolve().parent))
from _refenv import use_reference  # noqa: E402

TABLES = REPO / "lighthit_b200" / "tables"
OUT = REPO / "tests" / "golden" / "formats"
N_INT, N_OMEGA = 2, 4
PACK_INDICES = ((0, 16, 32, 64), (0, 1, 2, 3))  # frequency indices of the two pack bundles


def main():
    use_reference()
    from lighthit.band_fold import save_folded
    from lighthit.cache import CacheGrid, ResponseCache
    from lighthit.green import SolverSettings
    from lighthit.medium import Medium
    from lighthit.shower_basis import Ge2KernelStore
    if OUT.exists():
        shutil.rmtree(OUT)
    OUT.mkdir(parents=True)

    # the band-folded bundle of the README configuration (sliced)
    t = np.load(TABLES / "ge2_fold_48om_2-150m.npz")
    folded = dict(coefficients=np.ascontiguousarray(t["coefficients"][:, :N_INT, ..., :N_OMEGA]),
                  log_r=t["log_r"][:N_INT + 1], omega=t["omega"][:N_OMEGA],
                  absorption=t["absorption"], speed=t["speed"], degree=int(t["degree"]),
                  acceptance_degree=int(t["acceptance_degree"]),
                  pair_lambda=t["pair_lambda"], pair_mu=t["pair_mu"], phase=str(t["phase"]),
                  band_fold=dict(bands=[int(b) for b in t["bands"]], rank=len(t["bands"]),
                                 beta_design_min=0.75, worst_residual_design=1e-3,
                                 worst_residual_all=2e-3),
                  subdivide=1)
    save_folded(folded, OUT / "folded")

    # a per-wavelength kernel pack: two bundles (seeded coefficients, the
    # README kernel's near-field metadata)
    n = np.load(TABLES / "near_c0.npz")
    rng = np.random.default_rng(5)
    store = Ge2KernelStore(np.complex64)
    for b, indices in enumerate(PACK_INDICES):
        shape = (3, N_INT, int(n["degree"]) + 1, len(n["pair_lambda"]), 4, N_OMEGA)
        coef = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
        log_r = np.linspace(np.log(2.0), np.log(150.0), N_INT + 1)
        store._bundles[((f"table-{b}-a", f"table-{b}-b", f"table-{b}-c"), 8, indices)] = dict(
            coefficients=coef, degree=int(n["degree"]),
            acceptance_degree=int(n["acceptance_degree"]), pair_lambda=n["pair_lambda"],
            pair_mu=n["pair_mu"], omega=n["omega"][list(indices)], log_r=log_r,
            absorption=n["absorption"], speed=n["speed"], phase="flight")
    store.save(OUT / "pack")

    # the 450 nm flash cache (sliced radii and frequencies)
    f = np.load(TABLES / "flash_450nm_2-250m.npz")
    deg = int(f["degree"])
    grid = CacheGrid(f["radii_m"][:6], f["omega_per_ns"][:5])
    medium = Medium(float(f["absorption_per_m"]), float(f["scattering_per_m"]), float(f["g"]),
                    float(f["group_index"]), float(f["wavelength_nm"]))
    cache = ResponseCache(grid, medium, SolverSettings(spatial_degree=deg),
                          f["moments"][:5, :6], radial_phase=str(f["radial_phase"]))
    cache.save(OUT / "transport-450.npz")
    print("wrote", sorted(p.name for p in OUT.rglob("*") if p.is_file()))


if __name__ == "__main__":
    main()

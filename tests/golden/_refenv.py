"""Environment for the fixture scripts in this folder.

These scripts import the LightHit reference package (pure Python + Numba) in a
container where its source tree is present, run its own float64 routes and
write the results as small fixtures. They never run on a machine without the
reference; the tests only read the fixtures they wrote.
"""
import os
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[2]


def _required(name, what):
    value = os.environ.get(name)
    if not value:
        raise SystemExit(f"set {name} to {what}")
    return Path(value)


def __getattr__(name):
    """``REFERENCE_SRC`` and ``WORK``, read from the environment when first used."""
    if name == "REFERENCE_SRC":
        return _required("LIGHTHIT_REFERENCE_SRC", "the reference's src folder")
    if name == "WORK":
        return _required("LIGHTHIT_FIXTURE_WORK", "a writable folder for the reference's caches")
    raise AttributeError(name)


def use_reference():
    """Put the reference on ``sys.path`` with a writable Numba cache.

    Needs ``LIGHTHIT_REFERENCE_SRC`` (the reference's ``src`` folder) and
    ``LIGHTHIT_FIXTURE_WORK`` (a writable folder for its RTE caches; the Numba
    cache goes to ``NUMBA_CACHE_DIR``, or ``<work>/numba-cache`` when unset)."""
    REFERENCE_SRC, WORK = __getattr__("REFERENCE_SRC"), __getattr__("WORK")
    if not REFERENCE_SRC.exists():
        raise SystemExit(f"reference sources not found at {REFERENCE_SRC}")
    WORK.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("NUMBA_CACHE_DIR", str(WORK / "numba-cache"))
    if str(REFERENCE_SRC) not in sys.path:
        sys.path.insert(0, str(REFERENCE_SRC))
    import lighthit  # noqa: F401
    return lighthit


def table_work():
    """``LIGHTHIT_TABLE_WORK``: the folder where ``build_tables.py`` left the
    reference's RTE caches and kernel packs."""
    return _required("LIGHTHIT_TABLE_WORK", "the folder of build_tables.py's reference caches")

"""Environment for the fixture scripts in this folder.

These scripts import the LightHit reference package (pure Python + Numba) in a
container where its source tree is present, run its own float64 routes and
write the results as small fixtures. They never run on a machine without the
reference; the tests only read the fixtures they wrote.
"""
import os
import sys
from pathlib import Path

REFERENCE_SRC = Path(os.environ.get("LIGHTHIT_REFERENCE_SRC", "/root/reference/src"))
REPO = Path(__file__).resolve().parents[2]
WORK = Path(os.environ.get("LIGHTHIT_FIXTURE_WORK", REPO / "_work" / "ref"))


def use_reference():
    """Put the reference on ``sys.path`` with a writable Numba cache."""
    if not REFERENCE_SRC.exists():
        raise SystemExit(f"reference sources not found at {REFERENCE_SRC}")
    WORK.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("NUMBA_CACHE_DIR", str(REPO / "_work" / "numba-cache"))
    if str(REFERENCE_SRC) not in sys.path:
        sys.path.insert(0, str(REFERENCE_SRC))
    import lighthit  # noqa: F401
    return lighthit

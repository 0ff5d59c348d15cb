"""Command-line launcher: python ccs.py mol.xyz [--method pa|ehss|both] ...

Drop-in for the reference's ccs.py; the calculation runs on the B200 path
(ehss_b200.ccs_cli).
"""
import os
import sys
from pathlib import Path

for _name in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
    os.environ.setdefault(_name, "1")
sys.path.insert(0, str(Path(__file__).resolve().parent))

from ehss_b200.ccs_cli import main  # noqa: E402

if __name__ == "__main__":
    raise SystemExit(main())

"""Test infrastructure (oracle only): where the reference checkout is.

The location comes from the environment variable DEFMM_REFERENCE_DIR, else
from the default of oracle/Makefile (the recipe that builds the reference).
Returns None when no checkout is there (as on a machine that only runs the
prebuilt oracle/_ref files).
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_dir():
    d = os.environ.get("DEFMM_REFERENCE_DIR")
    if not d:
        try:
            cp = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True,
                                timeout=60)
            d = cp.stdout.strip()
        except (OSError, subprocess.SubprocessError):
            d = ""
    return d if d and os.path.isdir(os.path.join(d, "include")) else None

"""CPU oracle of the Schroedinger-Poisson hot path (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
as the checker; the product path never imports it.

REFERENCE_DIR is the one place that names where the reference source tree
lives on a build machine: the environment variable QX_REFERENCE_DIR, else the
default below.  It is read only to build oracle/_ref and to regenerate the
golden fixtures; nothing at test or bench time reads the reference tree.
"""
import os

REFERENCE_DIR = os.environ.get("QX_REFERENCE_DIR", "/root/reference")

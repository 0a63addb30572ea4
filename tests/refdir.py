"""Where the reference's source tree is, for the tests that read it (its example files and its
Python package): the directory in BRISK_REFERENCE_DIR, by default the read-only checkout of this
container.  Those tests are skipped where the tree is absent (the GPU box)."""
import os

REF_DIR = os.environ.get("BRISK_REFERENCE_DIR", "/root/reference")

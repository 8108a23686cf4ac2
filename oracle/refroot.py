"""Where the build recipes under oracle/ find the reference tree (test
infrastructure only): the directory named by $REF_ROOT, else the mount point
of the reference checkout in the build container. The recipes compile the
reference's sources from there into oracle/_ref/; nothing at run time reads
the tree (the GPU machines run the prebuilt files)."""
from __future__ import annotations

import os
from pathlib import Path

REF_ROOT = Path(os.environ.get("REF_ROOT") or "/root/reference")

"""Where the fixture scripts in this folder find the reference's sources:
the first command-line argument, else the CT2_REFERENCE_ROOT environment
variable.  Used at fixture-generation time only; the tests read the
committed .npz files."""
import os
import sys


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CT2_REFERENCE_ROOT")
    if not root or not os.path.isdir(os.path.join(root, "emil_code")):
        sys.exit("usage: %s <reference root containing emil_code/> "
                 "(or set CT2_REFERENCE_ROOT)" % os.path.basename(sys.argv[0]))
    return root

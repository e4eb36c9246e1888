"""Where the fixture generators of tests/golden/ find the reference checkout.

The path is the first command-line argument of a generator, else the
environment variable KERNELFORGE_REFERENCE_ROOT; there is no default, because
the checkout's location differs between machines.
"""
import os
import sys


def reference_root(argv):
    """The reference checkout named by argv[0] or KERNELFORGE_REFERENCE_ROOT."""
    root = argv[0] if argv else os.environ.get("KERNELFORGE_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: python <generator>.py REFERENCE_ROOT "
                 "(or set KERNELFORGE_REFERENCE_ROOT)")
    if not os.path.isdir(os.path.join(root, "src")):
        sys.exit(f"{root} does not look like a kernelforge checkout (no src/)")
    return root

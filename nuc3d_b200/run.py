"""``python -m nuc3d_b200.run RUNDIR``: see nuc3d_b200.rundir."""
import sys

from .rundir import main

if __name__ == "__main__":
    sys.exit(main())

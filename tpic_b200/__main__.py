"""`python -m tpic_b200 --run deck.inp --mass-matrix ...`: see tpic_b200.runner."""
import sys

from .runner import main

sys.exit(main())

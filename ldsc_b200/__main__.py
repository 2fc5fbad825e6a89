"""python -m ldsc_b200 l2 ... (the reference's `ldsc l2`)."""
import sys

from .cli import main

sys.exit(main())

"""``python -m 2d4_b200 ...``: the reference program's command line (cli.py)."""
import sys

from .cli import main

sys.exit(main())

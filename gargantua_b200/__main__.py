"""`python -m gargantua_b200 ...`: the command line in cli.py."""
import sys

from .cli import main

sys.exit(main())

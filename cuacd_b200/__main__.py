"""`python -m cuacd_b200 INPUT OUTPUT [options]`: the command-line pipeline
(cuacd_b200/cli.py)."""
import sys

if __name__ == "__main__":            # spawned workers import this module under another name
    from .cli import main
    sys.exit(main())

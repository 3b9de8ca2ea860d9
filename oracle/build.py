"""Build the CPU oracle library: python -m oracle.build [--force]."""
import sys

from .oracle import build

if __name__ == "__main__":
    print(build(force="--force" in sys.argv))

"""python -m transportse_b200 <config.py> [--steps N]: run a TRANSPORTSE config on the GPU."""
from .driver import main

if __name__ == "__main__":
    main()

"""CPU oracle of the Biot-Savart hot path (test infrastructure only; see oracle.py)."""

"""2D SIPG solve path: mesh setup, device operator, solves, multigrid."""

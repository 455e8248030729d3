"""B200 solver for the MELODY 2D explicit-dynamics step (see include/melgpu.h)."""

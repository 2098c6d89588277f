"""gfb -- host-side Python package of the B200 CG-SEM elastic solver."""

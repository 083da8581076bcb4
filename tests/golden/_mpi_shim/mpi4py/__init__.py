"""Single-rank mpi4py stand-in used only to import the upstream package for fixture generation."""

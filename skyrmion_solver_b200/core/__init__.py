"""Core engine: parameters, launchables, reductions, integrator and the Simulation driver."""

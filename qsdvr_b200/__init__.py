"""qsdvr_b200 — B200-native (sm_100a) QSDVR differentiable renderer hot path.

Modules:
  qsdvr   drop-in for the reference's ``qsdvr`` extension (14 ops + CameraArgs)
  render  the reference's autograd Functions, QuadricGrid and RenderGrid
  camera  per-camera ray tables and per-step sample lists
"""
__version__ = "0.1.0"

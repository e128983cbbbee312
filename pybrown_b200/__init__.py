"""pybrown_b200: B200-native (sm_100a) hydrodynamic hot path of pyBrown.

Drop-in modules mirroring the reference package layout:
  pybrown_b200.bead       -- Bead, pair vectors, overlap test (pyBrown.bead)
  pybrown_b200.diffusion  -- RPY / Smith-Ewald / Jeffrey-Onishi tensors (pyBrown.diffusion)
  pybrown_b200.box        -- Box.propagate on a device-resident state (pyBrown.box)
  pybrown_b200.io         -- JSON input, .str/.xyz/.enr/.rst files (pyBrown.input/output)
  pybrown_b200.bd         -- the BD.py and BD-restart.py drivers
and, without a counterpart in the reference:
  pybrown_b200.batch      -- many replicas advanced together (ReplicaBatch)
  pybrown_b200.serve      -- continuous batching of simulation requests (Server)
All compute goes through libpybrown_b200.so (include/pybrown_b200.h).
"""
__version__ = "0.2.0"

"""hashpoint: B200-native (sm_100a) HashPoint point searching and sampling.

Subpackages/modules:
  native  -- ctypes binding of the C ABI (include/hashpoint_b200.h) and its build
  ops     -- torch-tensor entry points over the C ABI
  synth   -- seeded synthetic scenes and cameras
"""

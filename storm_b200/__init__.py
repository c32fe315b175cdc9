"""storm_b200 -- B200-native mapping hot path of the SToRM read mapper.

  storm_b200.build   build recipe of libstormgpu.so and the storm-nucleotide / storm-color CLIs
  storm_b200.api     ctypes bindings of the C ABI (include/stormgpu.h)
  storm_b200.synth   seeded synthetic references and reads for the measured workloads
"""
__all__ = ["api", "build", "synth"]

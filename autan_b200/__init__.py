"""B200-native explicit Euler residual-and-update path of Autan (cell-centred finite volumes on
unstructured meshes): host set-up, the sm_100a CUDA kernels behind a C ABI, and a Python mirror of
the reference's DeviceStepper interface (physics/include/autan/physics/euler_device.hpp)."""

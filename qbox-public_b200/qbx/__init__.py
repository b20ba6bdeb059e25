"""B200-native Kohn-Sham electronic step behind the reference's class API.

``qbx.capi`` binds the CUDA library (libqbx.so, C ABI in include/qbx.h);
``qbx.systems`` defines the seeded synthetic workloads.
"""

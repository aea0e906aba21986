"""B200-native elliptic SIMP elastostatics (Plato Analyze hot path) over a C ABI.

The compute lives in platoanalyze_b200/lib/libplato_b200.so (CUDA, sm_100a); this package
holds the ctypes binding (`capi`, which raises ImportError when the library is missing),
the box-mesh generator front end (`mesh`), the Python mirror of the reference's elliptic
interfaces (`problem`), the benchmark workloads (`workloads`) and the build script (`build`).
"""

// Additions to Gonzales' Package.swift that make libgzg.so (the B200 traversal
// and wavefront library) available to libgonzales.  This is a fragment, not a
// whole manifest: merge each part into the corresponding list.
//
// 1. The system-library target (module map in Sources/gzg, copied from this
//    repository's swift/Sources/gzg):
//
//        .systemLibrary(name: "gzg", path: "Sources/gzg"),
//
// 2. "gzg" in the dependencies of the libgonzales target, beside "mojoKernel":
//
//        dependencies: [ ..., "mojoKernel", "gzg", ... ],
//
//    and the header search path in its swiftSettings:
//
//        .unsafeFlags(["-Xcc", "-I/opt/gonzales-b200/include"]),
//
// 3. The library in the linker settings of the gonzales executable and test
//    targets, beside -lmojo:
//
//        .unsafeFlags(["-L/opt/gonzales-b200/gonzales_b200", "-lgzg",
//                      "-Xlinker", "-rpath", "-Xlinker", "/opt/gonzales-b200/gonzales_b200"])
//
// 4. Sources/libgonzales/Accelerators/GzgBackend.swift from this repository's
//    swift/Sources/libgonzales/Accelerators.
//
// /opt/gonzales-b200 stands for wherever this repository is checked out and
// built (python gonzales_b200/build.py writes gonzales_b200/libgzg.so).

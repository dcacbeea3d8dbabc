// swift-tools-version: 6.0
// GargantuaCUDA: the sm_100a library's C ABI (include/gargantua.h) as a
// Swift system-library module, and gg-still, a small Swift host that
// renders one still through it (the flow of Still.swift:8-69).
//
// Build the library first (python -c "import __graft_entry__ as g;
// g.build()" at the repository root, which writes
// gargantua_b200/libgargantua_b200.so), then `swift build` here. No Swift
// toolchain is installed in the image this library is developed in, so
// this package has not been compiled there; the ABI it binds is exercised
// from C++ (gargantua_b200/cli) and Python (tests/).
//
// To put the module under gargantua's own package instead, copy
// GargantuaCUDA/ next to Sources/ShaderTypes, add
//   .systemLibrary(name: "GargantuaCUDA", path: "Sources/GargantuaCUDA"),
// to its targets, add "GargantuaCUDA" to the Gargantua target's
// dependencies, and give that target cSettings
// [.define("GG_WITH_HOST_SHADER_TYPES"), .headerSearchPath("../ShaderTypes/include")]
// so both modules share ShaderTypes' structs.
import PackageDescription

let library = "../gargantua_b200"

let package = Package(
    name: "GargantuaCUDA",
    products: [
        .library(name: "GargantuaCUDA", targets: ["GargantuaCUDA"]),
        .executable(name: "gg-still", targets: ["gg-still"]),
    ],
    targets: [
        .systemLibrary(name: "GargantuaCUDA", path: "GargantuaCUDA"),
        .executableTarget(
            name: "gg-still",
            dependencies: ["GargantuaCUDA"],
            path: "Sources/gg-still",
            linkerSettings: [.unsafeFlags(["-L\(library)", "-Xlinker", "-rpath", "-Xlinker", library])]
        ),
    ],
    swiftLanguageModes: [.v6]
)

// gg-still: one still through the GargantuaCUDA module, the flow of
// gargantua's Still.render (Still.swift:8-69) with the Metal passes
// replaced by gg_* calls: settle the default disk, splat it exactly,
// build the sweep tables for the camera, march in compensated FP32, tone
// map on the device and write a PNG. Usage: gg-still out.png [width height]
import Foundation
import GargantuaCUDA

func check(_ status: Int32, _ what: String) {
    if status != 0 {
        FileHandle.standardError.write("\(what): \(String(cString: gg_last_error()))\n".data(using: .utf8)!)
        exit(2)
    }
}

let args = CommandLine.arguments
let path = args.count > 1 ? args[1] : "still.png"
let width = UInt32(args.count > 3 ? Int(args[2]) ?? 960 : 960)
let height = UInt32(args.count > 3 ? Int(args[3]) ?? 540 : 540)

var ctx: OpaquePointer?
check(gg_context_create(0, 0, &ctx), "context")
defer { gg_context_destroy(ctx) }

// ParticleSystem + SimPass: seed, then STILL_SETTLE_STEPS substeps.
var particles: OpaquePointer?
let count: UInt32 = 1_000_000
check(gg_particles_create(ctx, count, 1, UInt32(PotentialPaczynskiWiita), &particles), "particles")
defer { gg_particles_destroy(particles) }
check(gg_particles_seed(particles), "seed")
check(gg_particles_step(particles, 300), "settle")

// Volume + SplatPass: exact deposit, resolve, clear.
var volume: OpaquePointer?
check(gg_volume_create(ctx, 128, &volume), "volume")
defer { gg_volume_destroy(volume) }
var splat = SplatUniforms()
splat.volumeSize = 128
splat.particleCount = count
splat.halfExtent = 30
splat.peakTemperature = 8000
splat.emissionScale = 5e-4
splat.exactDeposit = 1
splat.seed = simd_uint2(x: 1, y: 0)
check(gg_splat(particles, volume, &splat), "splat")

// MarchPass.uniforms for the default orbit camera (Camera.swift:4-33).
let azimuth: Float = 0.6, elevation: Float = 0.32, distance: Float = 52
let position = SIMD3<Float>(distance * cos(elevation) * cos(azimuth), distance * cos(elevation) * sin(azimuth),
                            distance * sin(elevation))
let forward = -position / (position * position).sum().squareRoot()
var right = SIMD3<Float>(forward.y, -forward.x, 0)
right /= (right * right).sum().squareRoot()
let up = SIMD3<Float>(right.y * forward.z - right.z * forward.y, right.z * forward.x - right.x * forward.z,
                      right.x * forward.y - right.y * forward.x)
func f3(_ v: SIMD3<Float>) -> simd_float3 { simd_float3(x: v.x, y: v.y, z: v.z, pad_w: 0) }
let tanHalf = tan(Float(50.0 * Double.pi / 180.0) * 0.5)
var u = MarchUniforms()
u.cameraPosition = f3(position)
u.cameraRight = f3(right)
u.cameraUp = f3(up)
u.cameraForward = f3(forward)
u.tanHalfFov = simd_float2(x: tanHalf * Float(width) / Float(height), y: tanHalf)
u.resolution = simd_uint2(x: width, y: height)
u.volumeHalfExtent = 30
u.opacityScale = 5e-4
u.starBrightness = 1.5
u.driftBudget = 1e-5
u.starSeed = 1
u.redshift = 1
u.bakeCapacity = 96
u.geodesic = GeodesicSettings(stepFactor: 0.02, stepMin: 0.02, stepMax: 0.5, captureRadius: 2.02, escapeRadius: 60,
                              stepCap: 4096, emptyStepFactor: 0.06, emptyStepMax: 1.5)
check(gg_tables_update(ctx, distance, &u), "sweep tables")  // DeflectionTables.update + apply

var targets: OpaquePointer?
check(gg_targets_create(ctx, width, height, &targets), "targets")
defer { gg_targets_destroy(targets) }
var counters = MarchCounters()
check(gg_march(ctx, volume, &u, targets, Int32(GG_PRECISION_COMPENSATED.rawValue), &counters), "march")

// Capture.write: the tone curve to sRGB8 on the device, then a PNG.
var present = PresentUniforms()
present.exposure = 1
present.driftBudget = 1e-5
var rgba = [UInt8](repeating: 0, count: Int(width * height * 4))
check(gg_tonemap(targets, &present, &rgba), "tone map")
check(gg_write_png(path, rgba, width, height), "png")
print("\(width) by \(height): \(counters.rays) rays, \(counters.captured) captured, \(counters.overDriftBudget) over budget -> \(path)")

/*
 * Every constant the per-frame compute uses, in geometrized units
 * (G = c = M = 1, lengths in units of the hole's mass).
 *
 * Symbols and values are the ones gargantua's constants table defines
 * (Sources/Oracle/Constants.swift:56-325, rendered to
 * Sources/Gargantua/Shaders/Constants.h:8-216); a CPU test compares every
 * value here with that table, so the kernels and the host agree on one set.
 * Float constants carry an f suffix and unsigned ones a u suffix so the
 * header reads the same from C, C++ and CUDA.
 */
#ifndef GARGANTUA_CONSTANTS_H
#define GARGANTUA_CONSTANTS_H

/* Geometry of the Schwarzschild hole. */
#define R_SCHWARZSCHILD (2.0f)          /* horizon */
#define R_PHOTON_SPHERE (3.0f)          /* circular photon orbit */
#define R_ISCO (6.0f)                   /* innermost stable circular orbit */
#define R_MARGINALLY_BOUND (4.0f)       /* marginally bound circular orbit */
#define B_CRITICAL (5.196152422706632f) /* 3 sqrt(3), the shadow radius */
#define WEAK_DEFLECTION_COEFFICIENT (4.0f)

/* Where rays and particles stop. */
#define R_CAPTURE (2.02f)               /* one percent above the horizon */
#define KERR_CAPTURE_MARGIN (0.05f)     /* above the Kerr outer horizon */
#define R_ESCAPE (60.0f)

/* The disk and the volume it is binned into. */
#define R_DISK_OUTER (24.0f)
#define R_FEED_INNER (20.0f)
#define DISK_SLAB_HALF_HEIGHT (6.0f)
#define VOLUME_HALF_EXTENT (30.0f)

/* Particle dynamics. */
#define SIM_DT (0.1f)
#define SIM_SUBSTEPS (2u)
#define DRAG_ALPHA (0.003f)
#define PLUNGE_SPEED_LIMIT (12.0f)
#define FEED_VELOCITY_DISPERSION (0.02f)
#define DISK_ASPECT (0.05f)
#define T_PEAK_DEFAULT (8000.0f)
#define ZERO_TORQUE_FLOOR (0.01f)
#define CIC_CORNERS (8u)

/* Blackbody colour table. */
#define BLACKBODY_T_MIN (1000.0f)
#define BLACKBODY_T_MAX (40000.0f)
#define BLACKBODY_TABLE_SIZE (256u)

/* Geodesic step policy. */
#define STEP_CAP_INTERACTIVE (256u)
#define STEP_CAP_STILL (4096u)
#define STEP_RADIUS_FACTOR (0.02f)
#define STEP_MIN (0.02f)
#define STEP_MAX (0.5f)
#define STEP_FACTOR_EMPTY_INTERACTIVE (0.1f)
#define STEP_MAX_EMPTY_INTERACTIVE (3.0f)
#define STEP_FACTOR_EMPTY_STILL (0.06f)
#define STEP_MAX_EMPTY_STILL (1.5f)
#define MARCH_THREADGROUP_WIDTH (8u)
#define MARCH_THREADGROUP_HEIGHT (8u)

/* Bake strategy. */
#define BAKE_SAMPLES (96u)
#define BAKE_SPACING_VOXELS (0.5f)
#define BAKE_FRAMES (4u)

/* Sweep tables outside the integration sphere. */
#define SWEEP_TABLE_SIZE (1024u)

/* Conserved-quantity drift budgets. */
#define DRIFT_BUDGET_INTERACTIVE (0.0001f)
#define DRIFT_BUDGET_STILL (1e-05f)

/* Shading. */
#define EXPOSURE_DEFAULT (1.0f)
#define EMISSION_SCALE (0.0005f)
#define GAS_SPEED_CEILING (0.85f)
#define BEAMING_DENSITY_FLOOR (40.0f)
#define VOLUME_OPACITY (0.0005f)
#define STAR_BRIGHTNESS (1.5f)

/* Stills and budgets. */
#define STILL_SETTLE_STEPS (600u)
#define STILL_TILE (128u)
#define COMMAND_BUFFER_BUDGET_MS (30.0f)
#define MEMORY_BUDGET_FRACTION (0.4f)
#define MEMORY_BUDGET_CAP_BYTES (3000000000u)

/* Host-side table sizes (Presets.swift:45, DeflectionTables.swift:28-29). */
#define INVERSE_CDF_COUNT (1024u)
#define SWEEP_SPHERE_INTERVALS (2048u)
#define SWEEP_CAMERA_INTERVALS (256u)

#endif

/*
 * pbs_layouts.h - C-compatible mirrors of the reference's plain data layouts, for
 * callers that exchange these structs with the dose library or with files the
 * reference writes.
 *
 * Each struct keeps the reference's member order, member types and size, so a
 * buffer of the reference's type can be reinterpreted as the mirror and back.
 * The reference declares them with C++ constructors and operators
 * (include/core/common.cuh:39-228); the mirrors are plain C.
 *
 *   PbsVec3f / PbsVec3i / PbsVec2f   vec3f / vec3i / vec2f   common.cuh:39-78   12 / 12 / 8 bytes
 *   PbsGrid                          Grid                    common.cuh:146-149 48 bytes
 *   PbsSource                        Source                  common.cuh:151-154 40 bytes
 *   PbsBeam                          Beam                    common.cuh:156-160 52 bytes
 *   PbsSubspotInfo                   SubspotInfo             common.cuh:163-217 56 bytes
 *   PbsCPBGrid                       CPBGrid                 common.cuh:220-228 40 bytes
 *   PbsDoseBinHeader                 header of the dose .bin files written by
 *                                    src/tests/wrapper_integration_test.cu:3850-3859
 *                                    (36 bytes, then float dose [Z][Y][X])
 *
 * Two more layouts cross the boundary as flat float arrays and are described where
 * they are used (subsecondpbs.h): the subspot table [L][M][5] = (dx, dy, w, sigma_x,
 * sigma_y) (raytracedicom_integration.h:47-52) and the rayweq volume, a 9-float
 * header [depth0, dstep, nDepth, y0, dy, ny, x0, dx, nx] then [nx][ny][nDepth]
 * depths (raytracedicom_integration.h:63-70).
 *
 * With PBS_REFERENCE_NAMES defined before inclusion, the reference's own type
 * names are declared as aliases of the mirrors.
 */
#ifndef SUBSECONDPBS_LAYOUTS_H
#define SUBSECONDPBS_LAYOUTS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct PbsVec3f { float x, y, z; } PbsVec3f;
typedef struct PbsVec3i { int x, y, z; } PbsVec3i;
typedef struct PbsVec2f { float x, y; } PbsVec2f;

/* Voxel grid: corner = centre of voxel (0,0,0), resolution = voxel size,
 * upper_corner = corner + (dims - 1) * resolution (carbonPBS/cudaCalDose.cpp:1954-1955),
 * dims = voxel counts (x, y, z). */
typedef struct PbsGrid {
    PbsVec3f corner, resolution, upper_corner;
    PbsVec3i dims;
} PbsGrid;

/* Beam source: source and isocentre positions, virtual-source x direction and
 * virtual source-axis distance. */
typedef struct PbsSource {
    PbsVec3f source_pos, iso_pos, vs_dir_x;
    float v_sad;
} PbsSource;

/* One pencil beam: source, beam direction and its x axis, energy (MeV/u),
 * transverse and longitudinal cut-offs and the energy's table index. */
typedef struct PbsBeam {
    PbsVec3f source, bmdir, bmxdir;
    float ene, trans_cutoff, longitudal_cutoff;
    int ene_idx;
} PbsBeam;

/* One subspot as the legacy fluence path reads it from the subspot table: offsets
 * on the reference plane, weight, sigmas, energy index, position and direction
 * in the patient frame, effective sigma and a validity flag (one byte, then
 * three bytes of padding, as the reference's bool member). */
typedef struct PbsSubspotInfo {
    float delta_x, delta_y, weight, sigma_x, sigma_y;
    int ene_idx;
    PbsVec3f position, direction;
    float effective_sigma;
    unsigned char is_valid;
    unsigned char pad_[3];
} PbsSubspotInfo;

/* Grid of the legacy fluence's CPB cells: corner, cell size, cell counts and the
 * number of energy layers. */
typedef struct PbsCPBGrid {
    PbsVec3f corner, resolution;
    PbsVec3i dims;
    int n_layers;
} PbsCPBGrid;

/* Header of a dose .bin file: dims (x, y, z), voxel spacing, origin; the float32
 * dose [Z][Y][X] (x fastest) follows. */
typedef struct PbsDoseBinHeader {
    int dims[3];
    float spacing[3];
    float origin[3];
} PbsDoseBinHeader;

#ifdef PBS_REFERENCE_NAMES
typedef PbsVec3f vec3f;
typedef PbsVec3i vec3i;
typedef PbsVec2f vec2f;
typedef PbsGrid Grid;
typedef PbsSource Source;
typedef PbsBeam Beam;
typedef PbsSubspotInfo SubspotInfo;
typedef PbsCPBGrid CPBGrid;
#endif

#ifdef __cplusplus
}
#endif

#endif /* SUBSECONDPBS_LAYOUTS_H */

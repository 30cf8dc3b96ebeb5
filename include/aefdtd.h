/* aefdtd.h — C ABI of the B200-native 3D FDTD time-stepping core.
 *
 * The reference exposes this path as the C++ class `FDTD`
 * (src/finite_differences/FDTD/core/fdtd_core.h:26-285) driven by the mode
 * functions FDTD_normal_incidence (src/finite_differences/FDTD/modes/
 * normal_incidence.cpp:161-607) and mode_default_fdtd
 * (src/finite_differences/FDTD/modes/default_fdtd.cpp:24-210), with sensors
 * (src/finite_differences/FDTD/core/sensors.h:87-171) and sources
 * (src/finite_differences/FDTD/core/sources.h:219-240) holding the FDTD
 * object by reference. The reference has no C ABI or FFI; every entry point
 * below names the reference call it replaces.
 *
 * Conventions
 *  - Plain pointers and sizes only. Every call returns aefdtd_status; no
 *    exception crosses the ABI. aefdtd_last_error() gives a message.
 *  - One owning host thread per handle. Device work of a handle is ordered
 *    on that handle's own CUDA stream.
 *  - Field arrays use the reference Grid3 layout: element (i,j,k) at
 *    i + j*Nx + k*Nx*Ny (src/common/grid.h:862-868), over the TOTAL grid
 *    (structure + pads + PML).
 *  - Lengths in metres, times in seconds, angular frequencies in rad/s.
 */
#ifndef AEFDTD_H
#define AEFDTD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AEFDTD_ABI_VERSION 2

typedef enum aefdtd_status {
    AEFDTD_OK = 0,
    AEFDTD_BAD_ARG = 1,     /* invalid descriptor, index or size */
    AEFDTD_OOM = 2,         /* device allocation or admission refused */
    AEFDTD_TIMEOUT = 3,     /* a bounded device or host wait ran out */
    AEFDTD_CUDA_ERROR = 4,  /* a CUDA runtime call failed */
    AEFDTD_NOT_READY = 5,   /* call out of order (e.g. step before setup) */
    AEFDTD_NO_DEVICE = 6    /* no CUDA device visible: there is no CPU path */
} aefdtd_status;

/* Driver orderings. NORMAL = "fdtd_normal" (normal_incidence.cpp:325-436):
 * E, E-plane injection, H, H-plane injection, sensor feed, R/T plane sums.
 * CUSTOM = "fdtd" (default_fdtd.cpp:156-204): E, source inject_E, H, sensor
 * feed, source inject_H. OBLIQUE = "fdtd_oblique_ARS", one in-plane
 * wavevector (FDTD_oblique_biphase_comp, oblique_biphase.cpp:29-330): two grids hold
 * the real and imaginary parts of a Bloch-periodic field; per step E of both
 * grids, Bloch_Wideband inject_E, H of both, inject_H, sensor feed (real
 * grid), R/T sums. The grid padding rules follow the FDTD constructor
 * (fdtd_core.cpp:158-251) for modes "NORM", "CUSTOM" and "OBL_PHASE" (no x/y
 * PML or pads; z pads raised to 5 by the oblique driver). */
typedef enum aefdtd_mode { AEFDTD_MODE_NORMAL = 0, AEFDTD_MODE_CUSTOM = 1, AEFDTD_MODE_OBLIQUE = 2 } aefdtd_mode;

/* FP64: bit-compatible operation order with the reference CPU core.
 * FP32: fields, CPML and dispersive state in FP32; coefficients generated in
 * FP64; DFT sensors accumulate in split precision; flux integration in FP64. */
typedef enum aefdtd_precision { AEFDTD_FP64 = 0, AEFDTD_FP32 = 1 } aefdtd_precision;

/* Field components, same order as EX_FIELD..HZ_FIELD (src/common/phys_constants.h:28-35). */
enum { AEFDTD_EX = 0, AEFDTD_EY, AEFDTD_EZ, AEFDTD_HX, AEFDTD_HY, AEFDTD_HZ };

/* Plane orientations, same meaning as NORMAL_X..NORMAL_ZM
 * (src/common/enum_constants.h:30-35). */
enum {
    AEFDTD_NORMAL_X = 0, AEFDTD_NORMAL_XM, AEFDTD_NORMAL_Y, AEFDTD_NORMAL_YM,
    AEFDTD_NORMAL_Z, AEFDTD_NORMAL_ZM
};

/* Faces in descriptor arrays: xm, xp, ym, yp, zm, zp. */
enum { AEFDTD_XM = 0, AEFDTD_XP, AEFDTD_YM, AEFDTD_YP, AEFDTD_ZM, AEFDTD_ZP };

#define AEFDTD_MAX_TERMS 8 /* per model family, per material (mat_lib files hold up to 6) */

/* Grid and boundary description: the FDTD constructor arguments
 * (fdtd_core.h:86-94) plus set_pml_* (fdtd_pml.cpp:457-497) and
 * set_tapering (fdtd_utils.cpp:915-918). */
typedef struct aefdtd_grid_desc {
    int32_t abi_version;   /* = AEFDTD_ABI_VERSION */
    int32_t mode;          /* aefdtd_mode */
    int32_t precision;     /* aefdtd_precision */
    int32_t nx, ny, nz;    /* structure cells, before pads and PML */
    int32_t nt;            /* planned number of steps (sensor tapering) */
    int32_t tapering;      /* Ntap: s-curve over the last Ntap steps */
    double dx, dy, dz;
    double dt;             /* time step; <= 0 means the mode drivers' rule
                              min(D)/(sqrt(3)c)*0.99*time_mod (normal_incidence.cpp:191) */
    double time_mod;
    int32_t pml[6];        /* PML cells per face */
    int32_t pad[6];        /* pad cells per face (raised to 5 on PML axes) */
    double pml_kappa[6];   /* kappa_max per face */
    double pml_sigma[6];   /* scale on 0.8(m+1)/(eta0*D) (fdtd_pml.cpp:445-447) */
    double pml_alpha[6];   /* alpha_max per face, S/m */
    int32_t pml_m;         /* sigma/kappa grading order; 0 -> 4 (fdtd_pml.cpp:309) */
    int32_t pml_ma;        /* alpha grading order; 0 -> 2 (fdtd_pml.cpp:310) */
    int32_t device;        /* CUDA device ordinal */
    int32_t dft_block;     /* K: time steps buffered per DFT-sensor block; 0 -> 64 */
} aefdtd_grid_desc;

/* Material: Material (src/materials/material.h:33-93) restricted to the
 * FDTD-compatible models: eps_inf plus Debye (ds, t0), Drude (wd, g),
 * Lorentz (A, O, G) and critical-point (A, O, P, G) terms
 * (src/materials/dielec_models.cpp:197-454). */
typedef struct aefdtd_material_desc {
    double eps_inf;
    int32_t n_debye, n_drude, n_lorentz, n_critpoint;
    double debye[AEFDTD_MAX_TERMS][2];
    double drude[AEFDTD_MAX_TERMS][2];
    double lorentz[AEFDTD_MAX_TERMS][3];
    double critpoint[AEFDTD_MAX_TERMS][4];
} aefdtd_material_desc;

/* Normal-incidence excitation and R/T analysis (normal_incidence.cpp:228-249,
 * 387-415, 442-570). polarization: 0 = "TE" (Ey), 1 = "TM" (Ex). */
typedef struct aefdtd_normal_desc {
    int32_t polarization;
    int32_t nl;
    double lambda_min, lambda_max;
} aefdtd_normal_desc;

/* Planar spectral Poynting sensor (Spect_Poynting, s_spec_power.cpp:32-119;
 * generate_fdtd_sensor, sensors.cpp:402-417). box: x1,x2,y1,y2,z1,z2 in
 * structure-grid cells, shifted by the structure origin and clamped as in
 * Sensor::link (sensors.cpp:196-230). */
typedef struct aefdtd_sensor_desc {
    int32_t orientation;   /* AEFDTD_NORMAL_* */
    int32_t box[6];
    int32_t nl;
    double lambda_min, lambda_max;
} aefdtd_sensor_desc;

/* Oscillator point/box source (Oscillator, sc_oscillator.cpp:34-84). */
typedef struct aefdtd_source_desc {
    int32_t orientation;   /* AEFDTD_NORMAL_*: X/XM -> Ex, Y/YM -> Ey, Z/ZM -> Ez */
    int32_t box[6];        /* structure-grid cells, as for sensors */
    double lambda_min, lambda_max;
} aefdtd_source_desc;

/* Total-grid geometry after construction (FDTD members Nx..zs_e, Dt). */
typedef struct aefdtd_dims {
    int32_t nx, ny, nz;
    int32_t xs_s, xs_e, ys_s, ys_e, zs_s, zs_e;
    int32_t n_materials;
    int32_t step;          /* tstep */
    double dt;
    size_t device_bytes;   /* device memory held by the handle */
} aefdtd_dims;

typedef struct aefdtd_sim aefdtd_sim;

/* ---- lifecycle -------------------------------------------------------- */

/* Replaces FDTD::FDTD(...) (fdtd_core.cpp:158-285) + alloc_DEBH/bootstrap
 * (fdtd_core.cpp:1073-1135) + set_pml_* + set_tapering. Allocates fields and
 * CPML state on the device. */
aefdtd_status aefdtd_create(const aefdtd_grid_desc *desc, aefdtd_sim **out);
/* Replaces FDTD::~FDTD (fdtd_core.cpp:287-303). */
aefdtd_status aefdtd_destroy(aefdtd_sim *sim);
aefdtd_status aefdtd_get_dims(const aefdtd_sim *sim, aefdtd_dims *out);
const char *aefdtd_last_error(const aefdtd_sim *sim);
const char *aefdtd_status_string(aefdtd_status status);

/* ---- structure and materials ----------------------------------------- */

/* Replaces FDTD::set_matsgrid (fdtd_utils.cpp:572-796): copies a structure
 * map of nx*ny*nz material indices (x fastest) into the grid and replicates
 * edge slices into pads and PML. */
aefdtd_status aefdtd_set_material_map(aefdtd_sim *sim, const uint32_t *map, size_t count);
/* Replaces FDTD::set_material (fdtd_utils.cpp:810-820): FDTD_Material
 * link_grid + set_base_mat (mats.cpp:394-464) with recursive-convolution
 * coefficients generated in FP64 (mats_RC.cpp:126-184, mats_const.cpp:71-80). */
aefdtd_status aefdtd_set_material(aefdtd_sim *sim, uint32_t index, const aefdtd_material_desc *mat);

/* Structure discretisation on the device (Structure::discretize,
 * structure.cpp:94-113, and Structure::index, structure.cpp:223-258, with the
 * primitives' index tests of structure_primitives.cpp). Operation kinds and
 * their parameters (p[]) follow the reference's structure-script functions
 * (lua_structure.cpp:292-548) after their argument conversions: */
enum {
    AEFDTD_OP_BLOCK = 0,        /* x1,x2,y1,y2,z1,z2 (Add_Block, :24-39) */
    AEFDTD_OP_LAYER = 1,        /* axis (0/1/2 as double), z1, z2 (Add_Layer, :317-339) */
    AEFDTD_OP_SPHERE = 2,       /* x, y, z, r (Add_Sphere, :484-499) */
    AEFDTD_OP_CYLINDER = 3,     /* x1,y1,z1,x2,y2,z2,r: axis end points (Add_Cylinder, :255-285) */
    AEFDTD_OP_CONE = 4,         /* x1,y1,z1 (base centre), x2,y2,z2 (apex), r (Add_Cone, :101-134) */
    AEFDTD_OP_ELLIPSOID = 5,    /* x, y, z, rx, ry, rz (Add_Ellipsoid, :291-312) */
    AEFDTD_OP_SIN_LAYER = 6,    /* z1, a1, z2, a2, px, phi_x, py, phi_y (Add_Sin_Layer, :449-478) */
    AEFDTD_OP_VECT_BLOCK = 7,   /* xO,yO,zO, xA,yA,zA, xB,yB,zB, xC,yC,zC (Add_Vect_Block, :505-566) */
    AEFDTD_OP_VECT_TRI = 8,     /* the twelve of VECT_BLOCK, then alp (Add_Vect_Tri, :572-601) */
    AEFDTD_OP_COATING = 9,      /* theta, phi (degrees), thickness, delta, origin material (Add_Coating, :45-95) */
    AEFDTD_OP_CONF_COATING = 10, /* thickness, delta (<= 0: 5 nm), origin material (Add_Conf_Coating, :140-248) */
    AEFDTD_OP_MESH = 11         /* x, y, z (recorded, unused as in the reference), scale, mesh number in
                                   aefdtd_structure_desc.meshes (Add_Mesh, :396-440) */
};
/* A triangle mesh as Add_Mesh reads it from an OBJ file (obj_file_load,
 * mesh_tools.h:103-152: quads split into (0,1,2) and (0,2,3)): vertex
 * coordinates before scaling, three 0-based vertex numbers per triangle. A
 * point inside the scaled vertices' box is inside the mesh when a ray from
 * it crosses the triangles an odd number of times (Moller-Trumbore,
 * ray_intersect.h:121-166). */
typedef struct aefdtd_mesh {
    const double *vertices;
    const int32_t *faces;
    int32_t n_vertices, n_faces;
} aefdtd_mesh;
typedef struct aefdtd_structure_op {
    int32_t kind;
    int32_t mat_index;
    double p[16];
} aefdtd_structure_op;
/* Structure-wide settings: default material, periodic images (loop) and
 * mirror flips (flip) per axis, the nominal lengths lx, ly, lz that both use
 * and that the coatings read, and the meshes that AEFDTD_OP_MESH refers to. */
typedef struct aefdtd_structure_desc {
    int32_t default_material;
    int32_t periodic[3];
    int32_t flip[3];
    int32_t n_meshes;
    double lengths[3];
    const aefdtd_mesh *meshes;
} aefdtd_structure_desc;
/* Tags every cell corner (i*dx, j*dy, k*dz) of an nx*ny*nz structure grid
 * with the material of the last operation containing it, else the default
 * material; writes the map to host memory (out_map, nx*ny*nz, x fastest)
 * and, when sim is not NULL, also installs it as aefdtd_set_material_map
 * does. At most 256 operations; coatings may nest 3 deep. A directional
 * coating needs delta > 0 and theta below 90 degrees (the reference's marches
 * would not end otherwise). */
aefdtd_status aefdtd_discretize(aefdtd_sim *sim, int32_t nx, int32_t ny, int32_t nz,
                                double dx, double dy, double dz,
                                const aefdtd_structure_op *ops, int32_t n_ops,
                                const aefdtd_structure_desc *desc, uint32_t *out_map, int32_t device);
/* aefdtd_discretize without flips: periodic[3] and lengths l[3] as in
 * aefdtd_structure_desc. */
aefdtd_status aefdtd_voxelize(aefdtd_sim *sim, int32_t nx, int32_t ny, int32_t nz,
                              double dx, double dy, double dz,
                              const aefdtd_structure_op *ops, int32_t n_ops,
                              int32_t default_material, const int32_t periodic[3],
                              const double lengths[3], uint32_t *out_map, int32_t device);

/* ---- excitation and sensors ------------------------------------------ */

/* Sets up the normal-incidence drive: Gaussian plane-wave pulse (ChpIn::
 * init_pulse, chpin.cpp:479-545) injected one-way at plane zs_e-1, the
 * plane-sum R/T sensors and their spectrum (normal_incidence.cpp:228-262).
 * Requires mode NORMAL and a material map with materials set. */
aefdtd_status aefdtd_setup_normal(aefdtd_sim *sim, const aefdtd_normal_desc *nd);
/* Oblique incidence at a fixed in-plane wavevector (FDTD_oblique_biphase_comp,
 * oblique_biphase.cpp:29-330): kx_in, ky_in are the driver's kx_in, ky_in
 * (rad/m in vacuum; the grids use k = k_in * n_sup). Sets up the wideband
 * Bloch plane wave (Bloch_Wideband, sc_bloch.cpp:23-285, 30001 spectral
 * lines, injected at the structure top z = zs_e), the Bloch phases of the
 * x/y wraps and the R/T sums. polarization: 0 = "TE", 1 = "TM". Requires
 * mode OBLIQUE and a material map with materials set. */
typedef struct aefdtd_oblique_desc {
    int32_t polarization;
    int32_t nl;
    double lambda_min, lambda_max;
    double kx_in, ky_in;
} aefdtd_oblique_desc;
aefdtd_status aefdtd_setup_oblique(aefdtd_sim *sim, const aefdtd_oblique_desc *od);
/* Spectra of the steps run so far (oblique_biphase.cpp:334-480): after the
 * driver's resizing of the wavelength range to the 89-degree limit, nl_out
 * wavelengths of 10 columns: lambda, incidence angle (degrees), |r_TE|,
 * arg r_TE, |r_TM|, arg r_TM, |t_TE|, arg t_TE, |t_TM|, arg t_TM (the columns
 * of the driver's obl_ file). out holds at most nl_max rows. */
aefdtd_status aefdtd_get_oblique_spectra(aefdtd_sim *sim, double *out, int32_t nl_max, int32_t *nl_out);
/* Per-step R/T sums of the steps run (steps x 18 doubles: the complex
 * BRsensorX..Z, RsensorX..Z, TsensorX..Z of the driver; BT equals BR). */
aefdtd_status aefdtd_get_oblique_series(aefdtd_sim *sim, double *out, size_t count);
/* Replaces generate_fdtd_source(...Oscillator) + Source::link (sources.cpp:252-283). */
aefdtd_status aefdtd_add_oscillator(aefdtd_sim *sim, const aefdtd_source_desc *src, int32_t *source_id);
/* Replaces generate_fdtd_sensor(...PLANAR_SPECTRAL_POYNTING) (sensors.cpp:402-417). */
aefdtd_status aefdtd_add_planar_sensor(aefdtd_sim *sim, const aefdtd_sensor_desc *sd, int32_t *sensor_id);

/* ---- time stepping ---------------------------------------------------- */

/* Advances n full steps in the mode's driver order (see aefdtd_mode): the
 * loop bodies of normal_incidence.cpp:325-436 / default_fdtd.cpp:156-204,
 * with FDTD::update_E/update_H (fdtd_core.cpp:1163-1335) as fused device
 * kernels. Launches are asynchronous on the handle's stream; the call
 * returns once they are queued (aefdtd_synchronize waits). */
aefdtd_status aefdtd_step(aefdtd_sim *sim, int32_t n);
aefdtd_status aefdtd_synchronize(aefdtd_sim *sim);
/* Zeroes fields, CPML and dispersive state and all sensor accumulators and
 * sets tstep to 0 (FDTD::reset_fields, fdtd_utils.cpp:855-881). */
aefdtd_status aefdtd_reset(aefdtd_sim *sim);

/* ---- results ---------------------------------------------------------- */

/* Copies one field component of the total grid (Nx*Ny*Nz values) into host
 * memory as double regardless of precision (replaces reading FDTD::Ex..Hz).
 * In mode OBLIQUE components 6..11 are Ex..Hz of the imaginary grid (the
 * reference's fdtd_i; its x/y ghost layers are not stored). */
aefdtd_status aefdtd_get_field(aefdtd_sim *sim, int32_t component, double *out, size_t count);
/* Overwrites one field component from host memory (checkpoint restore). */
aefdtd_status aefdtd_set_field(aefdtd_sim *sim, int32_t component, const double *in, size_t count);
/* Device pointer of a field component (precision's element type) for
 * zero-copy consumers on the same device; valid until aefdtd_destroy. */
aefdtd_status aefdtd_field_device_ptr(aefdtd_sim *sim, int32_t component, void **ptr);

/* Normal-incidence plane sums per completed step, 12 series of `steps`
 * values in this order: BRx BRy BRz Rx Ry Rz BTx BTy BTz Tx Ty Tz
 * (normal_incidence.cpp:255-259,387-415). */
aefdtd_status aefdtd_get_plane_sums(aefdtd_sim *sim, double *out, int32_t steps);
/* Normal-incidence spectra over nl wavelengths, 15 columns per wavelength:
 * lambda, r, t  (spectdata_norm, normal_incidence.cpp:510-522), then
 * |rx| arg(rx) |rx|^2 |ry| arg(ry) |ry|^2 |tx| arg(tx) Tx |ty| arg(ty) Ty
 * (spectdata_norm2, normal_incidence.cpp:534-567). */
aefdtd_status aefdtd_get_normal_spectra(aefdtd_sim *sim, double *out, int32_t nl);
/* Flux spectrum of a planar sensor: rsp_result per wavelength
 * (Spect_Poynting::treat, s_spec_power.cpp:44-119), FP64. */
aefdtd_status aefdtd_get_sensor_flux(aefdtd_sim *sim, int32_t sensor_id, double *out, int32_t nl);
/* Raw DFT accumulators of a planar sensor: 6 components (Ex..Hz) x span1 x
 * span2 x nl complex values as interleaved double (re, im), i fastest. */
aefdtd_status aefdtd_get_sensor_dft(aefdtd_sim *sim, int32_t sensor_id, double *out, size_t count);
aefdtd_status aefdtd_get_sensor_shape(aefdtd_sim *sim, int32_t sensor_id, int32_t *span1, int32_t *span2, int32_t *nl);

/* Box spectral Poynting sensor (Box_Spect_Poynting, s_spec_power.cpp:124-232):
 * planar spectral Poynting sensors on the six faces of the box (structure
 * cells x1,x2,y1,y2,z1,z2): xm on x1, xp on x2-1, ym, yp, zm, zp likewise,
 * each face created as by aefdtd_add_planar_sensor (one of the 8 planar
 * sensors per simulation per face). disabled: bits 0..5 = xm, xp, ym, yp, zm,
 * zp (Sensor::disable_*). The flux is the sum of the face fluxes in that
 * order (Box_Spect_Poynting::treat). */
typedef struct aefdtd_box_sensor_desc {
    int32_t box[6];
    int32_t nl;
    int32_t disabled;
    double lambda_min, lambda_max;
} aefdtd_box_sensor_desc;
aefdtd_status aefdtd_add_box_sensor(aefdtd_sim *sim, const aefdtd_box_sensor_desc *desc, int32_t *box_id);
aefdtd_status aefdtd_get_box_flux(aefdtd_sim *sim, int32_t box_id, double *out, int32_t nl);

/* Single-wavelength field sensors (s_fieldmap.cpp), fed after every step
 * like the planar sensors, with the step index t of the simulation:
 *   AEFDTD_MAP_PLANE (FieldMap, :289-461): a plane normal to X, Y or Z
 *     (the -M orientations give the same map) at the box's first index along
 *     the normal; acc(i,j) += e^{i w t Dt} F(i,j) for the three E components,
 *     or the H components when magnetic is set (FieldMap::set_mag_map; the H
 *     phase is also e^{i w t Dt}); with cumulative set
 *     (FieldMap::set_cumulative) F is first summed along the normal over the
 *     box. Output 3 x span2 x span1 complex.
 *   AEFDTD_MAP_BLOCK (FieldBlock, :28-228): every cell of the box,
 *     E with e^{i w t Dt}, H with e^{i w (t + 1/2) Dt}. Output 6 x span3 x
 *     span2 x span1 complex.
 *   AEFDTD_MAP_POINT (FieldPoint, :702-732): E at one cell (the box's first
 *     corner) after each step, as a time series: steps x 3 doubles (Ex, Ey,
 *     Ez) for the steps fed, at most the grid's nt.
 * F is the field interpolated to the cell node as for the planar sensors
 * (FDTD::local_E*, local_H*, fdtd_utils.cpp:457-507); w = 2 pi c / lambda.
 * The box is in structure cells and clamped to the grid as by Sensor::link
 * (sensors.cpp:196-230). Accumulation is FP64 in both precisions. At most 8
 * field sensors per simulation; not for batch members. */
enum {
    AEFDTD_MAP_PLANE = 0, AEFDTD_MAP_BLOCK = 1, AEFDTD_MAP_POINT = 2
};
typedef struct aefdtd_fieldmap_desc {
    int32_t kind;          /* AEFDTD_MAP_* */
    int32_t orientation;   /* AEFDTD_MAP_PLANE: AEFDTD_NORMAL_* */
    int32_t box[6];        /* x1, x2, y1, y2, z1, z2, structure cells */
    int32_t cumulative;    /* AEFDTD_MAP_PLANE: sum along the normal first */
    int32_t magnetic;      /* AEFDTD_MAP_PLANE: H instead of E */
    double lambda;         /* analysis wavelength (m); unused by AEFDTD_MAP_POINT */
} aefdtd_fieldmap_desc;
aefdtd_status aefdtd_add_fieldmap(aefdtd_sim *sim, const aefdtd_fieldmap_desc *desc, int32_t *map_id);
/* shape[4]: span1, span2, span3 (1 for plane maps and points), components
 * (3 or 6; for points 3 and span1 = the number of steps recorded so far). */
aefdtd_status aefdtd_get_fieldmap_shape(aefdtd_sim *sim, int32_t map_id, int32_t shape[4]);
/* Plane maps and blocks: components x span3 x span2 x span1 complex values
 * as interleaved double (re, im), i fastest; count = 2 x that product.
 * Points: steps x 3 doubles; count = 3 x steps. */
aefdtd_status aefdtd_get_fieldmap(aefdtd_sim *sim, int32_t map_id, double *out, size_t count);

/* Completion sensor in energy mode (CompletionSensor(coeff),
 * s_completion.cpp:20-24, 39-43, 121-130, 177-190; checked by the drivers at
 * normal_incidence.cpp:417-427 and default_fdtd.cpp:193-203). After every
 * step the sum of Ex^2 + Ey^2 + Ez^2 over the grid is kept. After each step t
 * with t % check_every == 0, once t + 1 >= 2 max(Nx, Ny, Nz), the run
 * completes when that sum is below coeff times its maximum so far; aefdtd_step
 * then returns after step t, later calls run no step, and the normal-mode
 * spectra use Nt = t steps (the driver's rule). coeff <= 0 turns it off;
 * check_every 0 -> 500 (the reference default, with coeff 1e-3). Not for batch
 * members. */
aefdtd_status aefdtd_set_completion(aefdtd_sim *sim, double coeff, int32_t check_every);
/* Completion sensor in FT mode (CompletionSensor(lmin, lmax, coeff, Np,
 * layout), s_completion.cpp:26-37, 45-121, 137-166, 246-361): n_points probe
 * cells on the structure faces named by layout (three letters, per axis x y z:
 * n none, d lower face, u upper face, b both; or "v" for the volume; unknown
 * layouts and "nnn" become "nnb"), each with a wavelength drawn in
 * [lambda_min, lambda_max]. Every step the probe's E is accumulated into a
 * running single-frequency transform; at a check the run completes when 90% of
 * the probes vary by at most coeff of their mean over the last
 * max(lambda)/c/Dt steps. The draws come from a std::mt19937 seeded with
 * seed (the reference draws from its global generator, seeded with the start
 * time or by seedp). check_every 0 -> 500. coeff <= 0 turns the sensor off. */
aefdtd_status aefdtd_set_completion_ft(aefdtd_sim *sim, double lambda_min, double lambda_max, double coeff,
                                       int32_t n_points, const char *layout, uint32_t seed, int32_t check_every);
/* done: 1 after completion; stop_step: t (or -1); ratio: energy mode, last /
 * largest energy at the last check; FT mode, the fraction of probes not yet
 * settled at the last check. */
aefdtd_status aefdtd_get_completion(aefdtd_sim *sim, int32_t *done, int32_t *stop_step, double *ratio);

/* Per-launch device timings of the most recent aefdtd_step call, measured
 * with CUDA events on the handle's stream: milliseconds spent in the E
 * half-step kernels, the H half-step kernels and the sensor kernels. */
aefdtd_status aefdtd_get_timings(aefdtd_sim *sim, double *e_ms, double *h_ms, double *sensor_ms);
/* enable: 0 off; 1 per phase (E, H, sensors; concurrent branches inside
 * each phase); 2 per work-item group: the groups of each half-step run one
 * after another on the handle's stream, each between two events. */
aefdtd_status aefdtd_enable_timing(aefdtd_sim *sim, int32_t enable);
/* After a timed aefdtd_step in mode 2: mean milliseconds per step of each
 * group (index half*5 + group; half 0 = E, 1 = H; groups interior, z-CPML,
 * dispersive, general, x/y-CPML) and the cells it updates per half-step.
 * n must be 10. */
aefdtd_status aefdtd_get_group_timings(aefdtd_sim *sim, double *ms, int64_t *cells, int32_t n);
/* The handle's CUDA stream (a cudaStream_t), for callers that order their
 * own device work or timing events with the simulation's kernels. */
aefdtd_status aefdtd_get_stream(aefdtd_sim *sim, void **stream);
/* Number of device kernel launches issued by this handle since creation. */
aefdtd_status aefdtd_get_launch_count(aefdtd_sim *sim, uint64_t *launches);
/* Free and total memory of device `device` (cudaMemGetInfo with that device
 * current), for callers that size groups of simulations by footprint (the
 * oblique driver's wavevector sweep, batches). No reference counterpart. */
aefdtd_status aefdtd_device_memory(int32_t device, size_t *free_bytes, size_t *total_bytes);
/* Copy bandwidth of a device over a buffer of `bytes` (half copied into the
 * other half `reps` times): read plus written bytes per second in GB/s. Over a
 * buffer smaller than the L2 it measures the L2 ceiling the batches are sized
 * for. No reference counterpart (a measurement aid). */
aefdtd_status aefdtd_probe_copy_bandwidth(int32_t device, size_t bytes, int32_t reps, double *gbs);
/* Test hooks of the bounded device waits (no reference counterpart; tests
 * only). AEFDTD_TEST_DFT_WAIT_CYCLES sets the bound, in SM cycles, of each
 * mbarrier wait in the FP32 tensor-core DFT (default 2^32, about 2 s);
 * AEFDTD_TEST_DFT_WITHHOLD_COPY (value 1) makes that kernel issue no phasor
 * copy, so its first wait runs out: each CTA then flags the error, frees its
 * tensor memory and returns, and the next synchronising call returns
 * AEFDTD_TIMEOUT. Value 0 restores normal operation; the handle stays usable
 * (aefdtd_reset, then step again). */
#define AEFDTD_TEST_DFT_WAIT_CYCLES 1
#define AEFDTD_TEST_DFT_WITHHOLD_COPY 2
/* The same for the staged interior half-steps (AEFDTD_TMA=1): the bound of
 * each of their mbarrier waits (default 2^32 cycles), and (value 1) a
 * producer that issues no tensor copy and arrives on no stage, so that the
 * consumers' first wait runs out; every CTA then raises its abort flag, the
 * producer waits (bounded) for its stages, and the next synchronising call
 * returns AEFDTD_TIMEOUT. */
#define AEFDTD_TEST_STAGED_WAIT_CYCLES 3
#define AEFDTD_TEST_STAGED_WITHHOLD_COPY 4
/* The same for the persistent batch launch (aefdtd_batch_opts.persistent),
 * set on a member before its batch builds the member's subset: the bound of
 * each wait on a neighbour's progress counter (default 2^31 cycles), and
 * (value 1) a launch in which the subset's first unit never reports its
 * progress, so that its neighbours' waits run out; every CTA then leaves at
 * its next wait and the advance returns AEFDTD_TIMEOUT. */
#define AEFDTD_TEST_PERSIST_WAIT_CYCLES 5
#define AEFDTD_TEST_PERSIST_WITHHOLD 6
aefdtd_status aefdtd_test_hook(aefdtd_sim *sim, int32_t what, int64_t value);

/* ---- batches: many simulations advanced together ----------------------
 *
 * No single reference counterpart: a batch runs what the reference runs as one
 * FDTD_normal_incidence/FDTD_Mode per simulation (normal_incidence.cpp:161-436)
 * for many simulations at once (parameter sweeps of periodic unit cells).
 * Members are ordinary simulations (created, given map, materials and
 * excitation as usual) without planar DFT sensors; normal-mode plane sums and
 * spectra are kept per member. A member is stepped only by its batch
 * (aefdtd_step on it returns AEFDTD_NOT_READY) and leaves it with
 * aefdtd_batch_remove or aefdtd_destroy. All members share precision,
 * material-id width and DFT block size. Member results are the same as
 * stepping each alone (FP64: bit-identical fields). */
typedef struct aefdtd_batch aefdtd_batch;

typedef struct aefdtd_batch_opts {
    int32_t abi_version;      /* = AEFDTD_ABI_VERSION */
    int32_t device;           /* CUDA device of the batch and its members */
    int64_t l2_budget_bytes;  /* device state per subset of members stepped together; 0 -> 48 MiB, < 0 -> no limit */
    int32_t tile_y;           /* tile height 2, 4 or 8 (0 -> 4) until autotuned */
    int32_t kchunk;           /* planes per work item (0 -> each simulation's heuristic) until autotuned */
    int32_t use_graphs;       /* < 0: no CUDA graphs (direct launches) */
    int32_t graph_steps;      /* steps per captured graph of a subset; 0 -> 32 */
    int32_t lanes;            /* most subsets running concurrently (1..8); 0 -> 2 until autotuned. With
                               * L2-sized subsets (l2_budget_bytes >= 0) a subset of b bytes runs beside
                               * at most 96 MiB / b - 1 others, so that they stay in L2 together */
    int32_t persistent;       /* 1: each subset's chunk of steps runs as ONE persistent cooperative launch
                               * (CTAs own bands x z-chunks of the members and wait only on their
                               * neighbours' progress counters, every wait bounded); 0: one launch per
                               * work-item group and half-step; the autotuner times both. Subsets
                               * holding an oblique member or a completion sensor always take the
                               * split launches. FP64 fields are bit-identical either way; plane sums
                               * are added per row band instead of per block (last bits differ). A
                               * wait that runs out makes the advance return AEFDTD_TIMEOUT and leaves
                               * the members part-way through a chunk: reset them before reuse. */
} aefdtd_batch_opts;

#define AEFDTD_BATCH_MAX_CLASSES 32
typedef struct aefdtd_batch_info {
    int32_t n_members, n_active, n_subsets, n_classes, n_lanes;
    int32_t n_persistent;     /* subsets on the persistent launch */
    int64_t cells;            /* total cells of the active members */
    int64_t member_bytes;     /* device memory held by all members */
    int64_t batch_bytes;      /* device memory held by the batch itself (work lists, argument arrays) */
    int64_t l2_budget_bytes;
    uint64_t launches;        /* kernel launches issued by the batch */
    int32_t class_key[AEFDTD_BATCH_MAX_CLASSES];     /* ceil(Nx/16)*1000 + ceil(Ny/16); < 0: one oblique member */
    int32_t class_tile_y[AEFDTD_BATCH_MAX_CLASSES];
    int32_t class_kchunk[AEFDTD_BATCH_MAX_CLASSES];
} aefdtd_batch_info;

aefdtd_status aefdtd_batch_create(const aefdtd_batch_opts *opts, aefdtd_batch **out);
aefdtd_status aefdtd_batch_destroy(aefdtd_batch *batch);
const char *aefdtd_batch_last_error(const aefdtd_batch *batch);
/* Adds a simulation with a budget of `steps` more time steps. Members carry
 * no planar DFT sensors or field maps. A member with a completion sensor
 * (set before it joins, either mode) finishes at its completion step; one in
 * oblique mode runs as a subset of its own (class key below zero). */
aefdtd_status aefdtd_batch_add(aefdtd_batch *batch, aefdtd_sim *sim, int32_t steps);
aefdtd_status aefdtd_batch_remove(aefdtd_batch *batch, aefdtd_sim *sim);
aefdtd_status aefdtd_batch_set_budget(aefdtd_batch *batch, aefdtd_sim *sim, int32_t steps);
/* Chooses per size class the tile height (2, 4, 8) and planes per work item
 * (4, 8), then the subset L2 budget (48 MiB, 96 MiB, none) and the number of
 * lanes (1, 2, 4), by timing trial segments on the device. Every member must
 * be at step 0; members are reset to step 0. */
aefdtd_status aefdtd_batch_autotune(aefdtd_batch *batch);
/* Advances every member with budget left by up to max_steps steps. Members
 * run in subsets, one subset after another; a subset stops early, after the
 * segment in which one of its members uses up its budget, so that callers can
 * retire it and admit others between calls. *steps_done: the most steps any
 * subset ran (0 when no member has budget left). Waits for the device before
 * returning. */
aefdtd_status aefdtd_batch_advance(aefdtd_batch *batch, int32_t max_steps, int32_t *steps_done);
/* Members whose budget is used up: up to cap handles in out, count in *n. */
aefdtd_status aefdtd_batch_finished(aefdtd_batch *batch, aefdtd_sim **out, int32_t cap, int32_t *n);
aefdtd_status aefdtd_batch_get_info(aefdtd_batch *batch, aefdtd_batch_info *info);

/* ---- serving: a request loop with continuous batching -----------------
 *
 * No reference counterpart (the reference runs one script per simulation).
 * Jobs are normal-incidence cells with a step budget; they queue on the host
 * and are admitted, in arrival order, while their estimated device footprint
 * fits the memory budget; admitted jobs run as members of one batch and are
 * retired (spectra kept, device memory freed) as soon as their budget is
 * used. A job's spectra are the same alone and in any mix. */
typedef struct aefdtd_server aefdtd_server;

enum { AEFDTD_JOB_QUEUED = 0, AEFDTD_JOB_RUNNING = 1, AEFDTD_JOB_DONE = 2, AEFDTD_JOB_FAILED = 3 };

typedef struct aefdtd_server_opts {
    int32_t abi_version;      /* = AEFDTD_ABI_VERSION */
    int32_t device;
    double hbm_fraction;      /* memory budget as a fraction of device memory; 0 -> 0.8 */
    int64_t budget_bytes;     /* > 0: explicit budget instead of hbm_fraction */
    int32_t max_active;       /* 0: no limit on running jobs */
    int32_t segment_steps;    /* steps per poll; 0 -> 256 */
    int32_t lookahead;        /* queued jobs that may pass one that does not fit; 0 -> 16 */
    int32_t reserved;
    aefdtd_batch_opts batch;  /* options of the batch (abi_version and device are set by the server;
                                 l2_budget_bytes as for a batch: 0 -> 48 MiB L2-sized subsets,
                                 < 0 -> no limit: one merged subset per size class) */
} aefdtd_server_opts;

typedef struct aefdtd_job_desc {
    const aefdtd_grid_desc *grid;           /* mode must be AEFDTD_MODE_NORMAL */
    const uint32_t *map;                    /* nx*ny*nz structure map, x fastest */
    size_t map_count;
    const aefdtd_material_desc *materials;  /* indexed by the map */
    int32_t n_materials;
    const aefdtd_normal_desc *normal;
    int32_t steps;                          /* step budget (the driver's Nt) */
    int32_t cc_step;                        /* completion check period (0 -> 500) */
    double cc_coeff;                        /* > 0: energy-mode completion sensor (auto_tsteps(Nt, cc_step,
                                               cc_coeff)); the job ends at its completion step */
} aefdtd_job_desc;

typedef struct aefdtd_job_info {
    int32_t state;            /* AEFDTD_JOB_* */
    int32_t steps;
    int64_t cells;            /* total grid cells (after admission) */
    int64_t est_bytes;        /* footprint estimate used for admission */
    int64_t bytes;            /* device bytes held while running */
    double t_submit, t_admit, t_done;   /* seconds since server creation; -1 if not yet */
    int32_t stop_step;        /* completion step t of a job with a completion sensor, else -1 */
    int32_t reserved;
} aefdtd_job_info;

typedef struct aefdtd_server_stats {
    int32_t submitted, queued, running, done, failed, reserved;
    int64_t budget_bytes, in_use_bytes, peak_bytes;
    double p50_s, p99_s, mean_s;   /* time to spectrum (submit -> done) of done jobs */
    double elapsed_s;              /* first submit -> last done */
    double sims_per_s, gcells_per_s;
} aefdtd_server_stats;

aefdtd_status aefdtd_server_create(const aefdtd_server_opts *opts, aefdtd_server **out);
aefdtd_status aefdtd_server_destroy(aefdtd_server *server);
const char *aefdtd_server_last_error(const aefdtd_server *server);
/* Copies the job description; no device work. */
aefdtd_status aefdtd_server_submit(aefdtd_server *server, const aefdtd_job_desc *job, int32_t *job_id);
/* Retires finished jobs, admits queued ones, advances one segment; *n_done:
 * jobs finished during the call. */
aefdtd_status aefdtd_server_poll(aefdtd_server *server, int32_t *n_done);
aefdtd_status aefdtd_server_job_info(aefdtd_server *server, int32_t job, aefdtd_job_info *info);
/* The 15-column spectra of a done job, as aefdtd_get_normal_spectra. */
aefdtd_status aefdtd_server_job_spectra(aefdtd_server *server, int32_t job, double *out, int32_t nl);
aefdtd_status aefdtd_server_get_stats(aefdtd_server *server, aefdtd_server_stats *stats);

/* ---- allocation-free diagnostics -------------------------------------- */

/* No counterpart in the reference: an entry point for callers that must not
 * allocate device memory (a process whose device memory is committed up
 * front, e.g. a batch or serving loop admitted to a fixed share of HBM).
 *
 * out[p*3 + c] = sum over the whole x-y plane planes[p] of weight * fields[c],
 * summed in FP64 in the same order as the stepping path's transmission-plane
 * sums (aefdtd_get_plane_sums slots 9..11 for plane zs_s). fields: host array
 * of 3 device pointers, each nx*ny*nz values (x fastest) of the given
 * precision on the current device; out: 3*n_planes doubles of device memory
 * on the current device. Kernels are enqueued on `stream` (a cudaStream_t,
 * NULL = default stream); the call does not wait for them.
 *
 * Calls no allocating routine. Its scratch is a fixed 96 KiB device array
 * held by every device that loads the library until exit, which caps a call
 * at AEFDTD_STATIC_MAX_PLANES planes: more returns AEFDTD_BAD_ARG with the
 * reason in errbuf (may be NULL). Every call resolves that array's address
 * on the current device; the first call on a device also loads the library's
 * device code there, so make it before any stream capture on the device.
 * All calls share the array, so calls that overlap on the device race. */
#define AEFDTD_STATIC_MAX_PLANES 64
aefdtd_status aefdtd_plane_sums_static(const void *const *fields, int32_t precision, int32_t nx, int32_t ny,
                                       int32_t nz, const int32_t *planes, int32_t n_planes, double weight,
                                       double *out, void *stream, char *errbuf, size_t errbuf_len);

#ifdef __cplusplus
}
#endif

#endif /* AEFDTD_H */

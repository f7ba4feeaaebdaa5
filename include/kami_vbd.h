/*
 * kami_vbd.h -- C ABI of the B200 Stable Cosserat Rods vertex-block-descent solver.
 *
 * This library replaces, for KamiSimulator's StableCosseratRods solver, the C++ calls
 * that StableCosseratRodsSolver makes into YarnBall::Sim and SDFBodyCollisionSolver.
 * Every entry point is extern "C", takes plain pointers and sizes, never throws, and
 * returns a kami_status.  kami_vbd_last_error_string() describes the last failure on
 * the calling thread.  Citations are file:line in the KamiSimulator project.
 *
 * Vertex order at the boundary: strands are contiguous, described by CSR offsets
 * strand_begin[0..S] (strand s owns vertices strand_begin[s] .. strand_begin[s+1]-1),
 * positions/velocities are packed float xyz triples in that order.  This is the
 * order of YarnBall::Sim::verts after createFromCurves (YarnBall/io/reader.cpp:16-50)
 * and of the rootVertices/strandRefs scatter in StableCosseratRodsSolver.cpp:238-277.
 * Internally the solver keeps its own tile-major layout on the device.
 */
#ifndef KAMI_VBD_H_
#define KAMI_VBD_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum kami_status {
    KAMI_OK = 0,
    KAMI_ERR_INVALID_ARGUMENT = 1, /* bad pointer, size, enum or parameter value */
    KAMI_ERR_CUDA = 2,             /* a CUDA runtime call failed (message has the CUDA error) */
    KAMI_ERR_OUT_OF_MEMORY = 3,    /* device or pinned-host allocation failed */
    KAMI_ERR_NONFINITE = 4,        /* the device status word saw a NaN/Inf position, velocity or orientation */
    KAMI_ERR_GEOMETRY = 5,         /* zero-length or dangling segment (Sim::configure, YBSimulator.cu:185-197) */
    KAMI_ERR_UNSUPPORTED = 6,      /* request outside what this library supports (e.g. strand longer than a tile) */
    KAMI_ERR_TIMEOUT = 7,          /* a bounded device wait gave up */
    KAMI_ERR_STATE = 8,            /* call made in the wrong order (e.g. backward without a recorded forward) */
    KAMI_ERR_CONTACTS = 9,         /* a segment had more than 16 hair-hair contacts (MAX_COLLISIONS_PER_SEGMENT,
                                      YarnBall.h:19; Sim::checkErrors throws there, YBSimulator.cu:396-398) */
    KAMI_ERR_IO = 10               /* a file could not be opened, read or written, or is not a USC .data file */
} kami_status;

/* Largest number of substeps (ceil(dt / max_h), Sim::advance, YarnBall/sim/step.cpp:38-62) one step
 * call takes; a dt above it is rejected with KAMI_ERR_INVALID_ARGUMENT. */
#define KAMI_MAX_SUBSTEPS 1000000

/* Gauss-Seidel order of the position and orientation sweeps. */
typedef enum kami_schedule {
    KAMI_SCHEDULE_COLOUR2 = 0, /* even then odd vertices, even then odd segments (by index within the strand) */
    KAMI_SCHEDULE_JACOBI = 1   /* all vertices from the previous sweep: the intent of cosseratItr /
                                  quaternionLambdaItr (YarnBall/sim/cosserat.cu:25-337), without their races */
} kami_schedule;

/* Which device implementation steps the solver. */
typedef enum kami_form {
    KAMI_FORM_AUTO = 0,  /* fused when every strand fits 8 warp tiles of 128 slots (1024 vertices) and
                            there is no hair-hair collision, else sweep */
    KAMI_FORM_SWEEP = 1, /* one kernel per colour sweep, replayed from a CUDA graph: the reference's
                            kernel-per-sweep structure (step.cpp:9-36), for hair-hair collision and
                            strands over 1024 vertices */
    KAMI_FORM_FUSED = 2  /* one kernel per step: each warp owns a strand tile for all iterations; strands
                            longer than a tile run on across the warps of a group of 2-8 tiles */
} kami_form;

typedef enum kami_stiffness_mode {
    KAMI_STIFFNESS_YOUNG = 0, /* Sim::setYoung(E [GPa], deviation), YBSimulator.cu:300-320 */
    KAMI_STIFFNESS_K = 1      /* Sim::setKStretch / setKBend, YBSimulator.cu:276-298 */
} kami_stiffness_mode;

typedef enum kami_memory {
    KAMI_MEMORY_HOST = 0,  /* pointer is host memory (pageable or pinned) */
    KAMI_MEMORY_DEVICE = 1 /* pointer is device memory of the solver's device */
} kami_memory;

/* Body signed-distance grid: SDFBodyCollisionSolver's grid (SDFBodyCollisionSolver.cpp:122-167,
 * cudaSDFCollision.cuh:23-48).  Node (i, j, k) sits at grid_min + ds * (i, j, k) with
 * ds = (grid_max - grid_min) / dims; arrays are x-fastest: index = i + nx * (j + ny * k). */
typedef struct kami_vbd_sdf_desc {
    int32_t dims[3];
    float grid_min[3];
    float grid_max[3];
    float threshold;   /* SDFThreshold: surface offset subtracted from phi (ThreshSdf) */
    const float* phi;  /* host, nx*ny*nz signed distances */
    const float* grad; /* host, 3*nx*ny*nz gradient (unnormalised) */
} kami_vbd_sdf_desc;

/* Everything StableCosseratRodsSolver::BuildYarnBallHair and JsonParams
 * (StableCosseratRodsSolver.h:41-112, .cpp:112-212) hand to YarnBall::Sim. */
typedef struct kami_vbd_desc {
    int32_t num_strands;
    const int32_t* strand_begin; /* host, num_strands + 1 CSR offsets; every strand >= 2 vertices */
    const float* positions;      /* host, 3 * V rest/initial positions [m] */
    const float* velocities;     /* host, 3 * V initial velocities [m/s], or NULL for zero */

    float radius;  /* MetaData::radius [m] */
    float density; /* [kg/m^3], Sim::configure(density) */

    int32_t stiffness_mode;        /* kami_stiffness_mode */
    float young;                   /* YoungsModule [GPa], used when strand_young is NULL */
    float deviation;               /* StiffnessDeviationCoeff, used when strand_deviation is NULL */
    const float* strand_young;     /* host, optional per-strand E [GPa] */
    const float* strand_deviation; /* host, optional per-strand bend/twist deviation (scales |qRest|) */
    float k_stretch;               /* StretchK (KAMI_STIFFNESS_K) */
    float k_bend;                  /* BendK (KAMI_STIFFNESS_K) */

    float gravity[3];                /* MetaData::gravity [m/s^2] */
    float damping;                   /* MetaData::damping (reference default 1e-6) */
    float velocity_decay;            /* VelocityDecay */
    float acceleration_ratio;        /* MetaData::accelerationRatio (1) */
    float external_force_multiplier; /* ExternalForceMultiplier */
    float wind_peak, wind_y_freq, wind_z_freq, wind_time_freq, wind_sharpness; /* Wind* (iteration.cu:19-29) */

    int32_t num_itr;   /* NumItr: VBD iterations per substep */
    float max_h;       /* Sim::maxH: substeps = ceil(dt / max_h) (step.cpp:42); reference fixes 4e-4 */
    int32_t schedule;  /* kami_schedule */
    int32_t form;      /* kami_form */
    int32_t pin_roots; /* 1: invMass = 0 at each strand root (StableCosseratRodsSolver.cpp:203-205) */
    int32_t device;    /* CUDA device ordinal; -1 = current device */

    const kami_vbd_sdf_desc* sdf; /* NULL: no body collision (EnableSDF false) */

    /* Device tile shape (no counterpart in the reference; 0 = automatic).  slots_per_lane: even C,
     * each warp tile holds 32*C vertex slots (the fused form supports C = 2 and 4, and puts strands
     * longer than a tile into groups of as many tiles as they need, up to 8);
     * warps_per_block: warps per CTA of the fused kernel. */
    int32_t slots_per_lane;
    int32_t warps_per_block;

    /* Hair-hair collision: EnableHairHairColl (StableCosseratRodsSolver.cpp:176-186) with the
     * MetaData constants of YarnBall.h:93-114.  Runs on the sweep form (form AUTO picks it).
     * Contacts are detected every detection_period substeps from the predicted motion and resolved
     * with an IPC barrier plus friction inside the position sweeps; a segment holds at most 16. */
    int32_t hair_hair;         /* 1: on */
    float barrier_thickness;   /* barrierThickness [m]; the solver sets 2 (1 - 0.05) CurveRadius */
    float k_collision;         /* kCollision (1e-5) */
    float k_friction;          /* kFriction (5) */
    float friction_coeff;      /* frictionCoeff (0.1) */
    float detection_scaler;    /* detectionScaler (1.2), must be > 1 */
    int32_t detection_period;  /* detectionPeriod: substeps between detections (1); <= 0 never detects */
    int32_t step_limit;        /* useStepSizeLimit (1, as the solver sets it with EnableHairHairColl) */
    int32_t velocity_radius;   /* useVelocityRadius (1) */

    /* SagFreeItr: passes of sag-free initialisation run at creation, after root pinning, as
     * BuildYarnBallHair does (StableCosseratRodsSolver.cpp:208; Sim::SagFree, YBSimulator.cu:480-674);
     * 0 = none.  kami_vbd_sag_free runs it on demand. */
    int32_t sag_free_itr;

    /* Connection springs: Vertex::connectionIndex (YarnBall.h:56), the spring of stiffness 40 that
     * cosseratItr adds to a vertex tied to another one (cosserat.cu:123-131), as YarnBall sets it for
     * glued endpoints (jsonBuilder.cpp:165-185) and the two ends of a closed curve (reader.cpp:40-44).
     * host, one entry per vertex: the vertex of the same groom it is tied to (both ways for a mutual
     * tie), or -1; NULL = none.  The partner's displacement is read as it stood at the start of the
     * iteration (colour2: a snapshot taken per iteration, as hair-hair partners are; jacobi: the
     * previous iterate), where the reference reads it while other threads write it.  With hair-hair
     * collision, a pair of segments joined by a tie is not a contact (collision.cu:47-48; tested
     * from either segment).  Handles with a tie run on the sweep form (form AUTO picks it; FUSED and
     * a later change of the tile shape are KAMI_ERR_UNSUPPORTED). */
    const int32_t* connection_index;
} kami_vbd_desc;

typedef struct kami_vbd_solver* kami_vbd_handle;

/* Fills d with the reference's defaults (JsonParams(), StableCosseratRodsSolver.h:86-111, with
 * WindPeak 0 and max_h 4e-4) and zero/NULL geometry.  Replaces: JsonParams::JsonParams. */
kami_status kami_vbd_desc_init(kami_vbd_desc* d);

/* Builds the solver: flags, rest lengths, masses, orientations, rest Darboux quaternions and
 * stiffness, then uploads the state.
 * Replaces: YarnBall::createFromCurves (reader.cpp:16-50) + Sim::Sim (YBSimulator.cu:81-127) +
 * Sim::configure (YBSimulator.cu:161-274) + setYoung/setKStretch/setKBend (:276-320) + root
 * pinning (StableCosseratRodsSolver.cpp:203-209) + SDFBodyCollisionSolver::Construct (:11-21). */
kami_status kami_vbd_create(const kami_vbd_desc* desc, kami_vbd_handle* out);

/* Batched form: one handle over num_grooms independent grooms (descs[0..num_grooms-1]).  Their
 * strands are packed together into warp tiles, so one launch steps every groom.  Each groom's
 * material (masses, rest lengths, orientations, stiffness, root pinning and the set's last-vertex
 * flags) is set up exactly as kami_vbd_create would set it up for that groom alone.  The grooms
 * must agree on the solver-wide settings (gravity, damping, decay, acceleration ratio, external
 * force multiplier, wind, num_itr, max_h, schedule, form, device, tile shape, SDF); they may
 * differ in geometry, radius, density and stiffness.  At the boundary the grooms' vertices follow
 * one another in groom order (kami_vbd_batch_groom_range).  Replaces: one YarnBall::Sim per groom
 * stepped in sequence (the CantileverTestSolver pattern). */
kami_status kami_vbd_batch_create(int32_t num_grooms, const kami_vbd_desc* descs, kami_vbd_handle* out);

/* Number of grooms of a handle (1 for kami_vbd_create). */
kami_status kami_vbd_batch_count(kami_vbd_handle h, int32_t* num_grooms);

/* Where groom `groom` sits in the handle's boundary order: its first strand and strand count, its
 * first vertex and vertex count (any output may be NULL). */
kami_status kami_vbd_batch_groom_range(kami_vbd_handle h, int32_t groom, int32_t* strand_begin, int32_t* num_strands,
                                       int64_t* vertex_begin, int64_t* num_vertices);

/* Steps every groom of the handle n times: kami_vbd_step_n (persistent multi-step launches
 * replayed from a CUDA graph). */
kami_status kami_vbd_batch_step(kami_vbd_handle h, float dt, int32_t n, const float* body_transforms, void* stream);

/* Releases every device and host resource of the handle.  Replaces: Sim::~Sim (YBSimulator.cu:129-157). */
kami_status kami_vbd_destroy(kami_vbd_handle h);

/* Number of vertices / strands at the boundary, and the device-side tile shape (slots per lane). */
kami_status kami_vbd_get_sizes(kami_vbd_handle h, int64_t* num_vertices, int32_t* num_strands, int32_t* slots_per_lane);

/* Positions and velocities (3*V floats each, either may be NULL to leave it unchanged).
 * Replaces: StableCosseratRodsSolver::UploadHair -> Sim::uploadPosAndVel (.cpp:238-256,
 * YBSimulator.cu:375-380).  Last velocities and orientations are left untouched, as there. */
kami_status kami_vbd_set_positions_velocities(kami_vbd_handle h, const float* xyz, const float* vxyz, int32_t memory);

/* Replaces: StableCosseratRodsSolver::DownloadHair -> Sim::downloadPosAndVel (.cpp:258-277,
 * YBSimulator.cu:382-386).  Synchronises the solver's stream and reports KAMI_ERR_NONFINITE if the
 * device status word was raised since the last check. */
kami_status kami_vbd_get_positions_velocities(kami_vbd_handle h, float* xyz, float* vxyz, int32_t memory);

/* One frame of the plugin's host loop from host buffers to host buffers: UploadHair, SolveNextStep(dt),
 * DownloadHair (StableCosseratRodsSolver.cpp:216-277, i.e. Sim::uploadPosAndVel, Sim::advance and
 * the SDF pass, Sim::downloadPosAndVel).  The result is that of kami_vbd_set_positions_velocities,
 * kami_vbd_step and kami_vbd_get_positions_velocities with host memory (3*V floats per array;
 * xyz_out / vxyz_out may be xyz / vxyz).  With the fused form, no hair-hair collision and all four
 * arrays each inside one page-locked host allocation mapped into the device's address space
 * (cudaHostAlloc / cudaMallocHost, pinned torch tensors), the frame is one kernel launch: each warp
 * reads its tile's strands from the host buffers, steps them and writes them back, so both PCIe
 * directions overlap the arithmetic of other tiles and no copy engine or staging pass is involved.
 * Otherwise the three calls run in turn.  Blocks until the outputs are written; reports
 * KAMI_ERR_NONFINITE as kami_vbd_get_positions_velocities does. */
kami_status kami_vbd_step_host(kami_vbd_handle h, float dt, const float* xyz, const float* vxyz, float* xyz_out,
                               float* vxyz_out);

/* Segment orientations (4*V floats, x y z w per vertex; the tip copies its previous segment).
 * Replaces: the qs part of Sim::download (YBSimulator.cu:355-360). */
/* Hair preprocessing that StableCosseratRodsSolver runs before it builds the simulation, on the
 * GPU (one thread per strand), over padded [strand][max_verts] xyz arrays in host memory.
 * kami_hair_subdivide = Kami::HairMods::DivideHair (utilities/HairModification.cpp:12-80), SubdivCoeff
 * = mul: mul - 1 evenly spaced points inserted into every segment of positions (and velocities,
 * when given); output rows of (max_verts - 1) * mul + 1 (out_* rows beyond a strand's end keep
 * their values); out_counts = (count - 1) * mul + 1.
 * kami_hair_resample = BuildYarnBallHair's EnableResample step (StableCosseratRodsSolver.cpp:141-163,
 * Resample::resampleCMR in YarnBall/io/resample.h): each strand of >= 4 points is resampled, in
 * place, along its Catmull-Rom spline to segments of target_len (from its 2nd to its next-to-last
 * point), subsampled to max_verts when longer; counts are updated; shorter strands are left as they
 * are.  Results equal the reference's to the bit (the file is compiled without FMA contraction). */
kami_status kami_hair_subdivide(int32_t num_strands, const int32_t* counts, int32_t max_verts, const float* xyz,
                                const float* vxyz, int32_t mul, int32_t* out_counts, float* out_xyz, float* out_vxyz,
                                int32_t device);
kami_status kami_hair_resample(int32_t num_strands, int32_t* counts, int32_t max_verts, float* xyz, float target_len,
                               int32_t device);

/* Sag-free initialisation (Sim::SagFree, YBSimulator.cu:480-674) on the GPU, one thread per strand:
 * rest lengths that cancel the stretch force of the hanging mass, and orientations / rest Darboux
 * turned to cancel the bending torque under the handle's gravity, `iterations` passes.  Positions
 * are unchanged.  Call it before stepping, as the reference does at construction. */
kami_status kami_vbd_sag_free(kami_vbd_handle h, int32_t iterations);

/* Device-resident Hair.  KamiSimulator's Hair keeps positions and velocities in padded
 * [strand][vertex] arrays: xyz of Hair strand u, vertex v at (u * max_verts + v) * 3
 * (EigenVecX3f2DArray, LinearUtil.cpp:159, :247-253).  kami_vbd_set_hair_layout tells the solver
 * which Hair strand each of its strands is (strand_refs[s], NULL = identity; strands of fewer than 4
 * vertices are not in the solver, StableCosseratRodsSolver.cpp:134-136).  Then
 * kami_vbd_upload_hair / kami_vbd_download_hair replace UploadHair / DownloadHair
 * (StableCosseratRodsSolver.cpp:238-277) with one gather/scatter kernel over the padded arrays:
 * with device arrays nothing crosses PCIe; with host arrays inside page-locked allocations mapped
 * into the device's address space (cudaHostAlloc, or kami_host_register) the kernel reads or writes
 * the host arrays itself, only the entries the solver owns; with other host arrays each array is
 * copied whole (download copies it in and out, so the entries the solver does not own keep their
 * values). */
kami_status kami_vbd_set_hair_layout(kami_vbd_handle h, int32_t hair_strands, int32_t max_verts,
                                     const int32_t* strand_refs);
kami_status kami_vbd_upload_hair(kami_vbd_handle h, const float* xyz, const float* vxyz, int32_t memory);
kami_status kami_vbd_download_hair(kami_vbd_handle h, float* xyz, float* vxyz, int32_t memory);

/* One frame of the plugin over the padded Hair arrays of kami_vbd_set_hair_layout: UploadHair from
 * hair_xyz_in / hair_vxyz_in (both NULL: the device state is current), SolveNextStep(dt) and
 * DownloadHair to hair_xyz_out / hair_vxyz_out (both NULL: the results stay on the device); outputs
 * may be the inputs.  StableCosseratRodsSolver.cpp:216-277 and KamiSimulator.cpp:380-390 in one call.
 * With the fused form, no hair-hair collision and every given array inside one page-locked mapped
 * allocation, it is one kernel launch that reads each tile's strands from the Hair, steps them and
 * writes them back (the fused_frame kernel of kami_vbd_step_host); otherwise the three calls run in
 * turn.  Blocks until the kernel has finished with the host arrays. */
kami_status kami_vbd_step_hair(kami_vbd_handle h, float dt, const float* hair_xyz_in, const float* hair_vxyz_in,
                               float* hair_xyz_out, float* hair_vxyz_out);

/* Page-locks and maps an existing host range (cudaHostRegister, mapped and portable) so that the
 * calls above take their one-launch paths on it, e.g. a Hair's arrays; kami_host_unregister undoes
 * it.  The range must stay allocated while registered.  No counterpart in the reference. */
kami_status kami_host_register(void* p, size_t bytes);
kami_status kami_host_unregister(void* p);

/* Body SDF grid baked from a closed, consistently wound triangle mesh on the GPU.  Replaces the
 * CPU bake of PNMesh::GenerateSDF + StoreSDFQueries (PNMesh.cpp:100-173; Discregrid in
 * utilities/Geometry.cpp:5-35).  Node (i, j, k) sits at grid_min + ds (i, j, k), ds = (grid_max -
 * grid_min) / dims, x fastest, as kami_vbd_sdf_desc expects.  phi: the exact signed distance to the
 * mesh (negative inside; sign by the angle-weighted pseudonormal of the nearest feature, as
 * Discregrid's TriangleMeshDistance decides it) -- the function the reference's cubic Lagrange grid
 * approximates.  grad (3 per node): inside, the unit gradient of the distance; elsewhere the unit
 * direction from the grid centre, StoreSDFQueries' choice for nodes at distance >= 0 (zero at a
 * node exactly at the centre).  The reference samples its grid over the mesh's bounding box.
 * memory: phi/grad in host or device memory; device: CUDA ordinal, -1 = current. */
kami_status kami_sdf_bake(const float* vertices, int32_t num_vertices, const int32_t* triangles, int32_t num_triangles,
                          const int32_t dims[3], const float grid_min[3], const float grid_max[3], float* phi,
                          float* grad, int32_t memory, int32_t device);

/* USC-HairSalon .data files (importers/USCHairsalonImporter.cpp:56-80, exporters/
 * USCHairsalonExporter.cpp:6-18): uint32 strand count, then per strand a uint32 vertex count and
 * that many float xyz triples.  kami_usc_info reads the strand table.  kami_usc_read fills
 * strand_vert_count[num_strands] and xyz, packed in strand order (max_verts = 0) or padded to
 * [strand][max_verts] like the Hair arrays (the reference's full import uses 100).  kami_usc_write
 * writes the same layouts; unlike ExportUSCHairCore it takes the full path (no ".data" appended).
 * Malformed or truncated files return KAMI_ERR_IO. */
kami_status kami_usc_info(const char* path, int32_t* num_strands, int64_t* num_vertices, int32_t* max_strand_verts);
kami_status kami_usc_read(const char* path, int32_t max_verts, int32_t* strand_vert_count, float* xyz);
kami_status kami_usc_write(const char* path, int32_t num_strands, const int32_t* strand_vert_count, int32_t max_verts,
                           const float* xyz);

kami_status kami_vbd_get_orientations(kami_vbd_handle h, float* xyzw, int32_t memory);
kami_status kami_vbd_set_orientations(kami_vbd_handle h, const float* xyzw, int32_t memory);

/* Rest Darboux quaternions scaled by the bend/twist stiffness (4*V floats), d_qRests of
 * YBSimulator.cu:256 after setYoung.  set_ lets a caller change bend/twist stiffness per vertex. */
kami_status kami_vbd_get_rest_darboux(kami_vbd_handle h, float* xyzw, int32_t memory);
kami_status kami_vbd_set_rest_darboux(kami_vbd_handle h, const float* xyzw, int32_t memory);

/* Body transform used by the SDF pass: rotation quaternion (x, y, z, w) and translation, as
 * SDFSimulationParams.rotation / translate (cudaSDFCollision.cuh:43-44, set in
 * SDFBodyCollisionSolver::SendSimParamsToCuda, .cpp:308-325). */
kami_status kami_vbd_set_body_transform(kami_vbd_handle h, const float rotation_xyzw[4], const float translate[3]);

/* One KamiSimulator internal step: Sim::advance(dt) (step.cpp:38-62) -- ceil(dt/max_h) substeps of
 * predict, num_itr x (position sweep, orientation sweep), velocity update -- followed by the SDF
 * body-collision pass that StableCosseratRodsSolver::SolveNextStep runs after it (.cpp:216-234),
 * with no host round trip.  Asynchronous on `stream` (a cudaStream_t; NULL = the handle's stream). */
kami_status kami_vbd_step(kami_vbd_handle h, float dt, void* stream);

/* Waits for the handle's work and checks the device status word.  Replaces: Sim::checkErrors
 * (YBSimulator.cu:388-414). */
kami_status kami_vbd_synchronize(kami_vbd_handle h);

/* Strain limiting: SDFBodyCollisionSolver's StrainLimiting kernel (SDFCollisionSolver/
 * cudaSDFCollision.cu:176-199), which the reference's SDF solver runs after its SDF pass when
 * UseStrainLimiting is set (SDFBodyCollisionSolver.cpp:186).  For every strand, from the root to the
 * tip, a segment whose length l differs from its rest length l0 by more than strain_error * l0 has
 * its far vertex moved along the segment by (l - l0), towards the near vertex as already corrected.
 * Positions only: velocities are left as they are.  l0 is the handle's rest length of the segment
 * (the segment's initial length, as the SDF solver's restLengthsVec, SDFBodyCollisionSolver.cpp:
 * 107-121).  Call it after kami_vbd_step, once per step, as the reference runs it once per
 * SolveNextStep; the reference's StrainError defaults to 0.1 (SDFBodyCollisionSolver.h:26).
 * strain_error must be finite and >= 0.  It has no adjoint: while the tape holds recorded steps it
 * returns KAMI_ERR_STATE.  Stream-ordered like kami_vbd_step.  The first call after creation or a
 * change of the tile shape builds a table of 12 bytes per strand on the device (a synchronising
 * allocation); later calls allocate nothing. */
kami_status kami_vbd_strain_limit(kami_vbd_handle h, float strain_error, void* stream);

/* Full dynamic state snapshot (positions, velocities, last velocities, orientations and the
 * h / lastH / time clock) for checkpoint/resume; the reference saves none of these. */
kami_status kami_vbd_state_size(kami_vbd_handle h, size_t* bytes);
kami_status kami_vbd_get_state(kami_vbd_handle h, void* dst, size_t bytes, int32_t memory);
kami_status kami_vbd_set_state(kami_vbd_handle h, const void* src, size_t bytes, int32_t memory);

/* ---- batched stepping and tile shape (no counterpart in the reference) -------------------------
 * One handle may hold many grooms (concatenate their strands): every strand is packed into warp
 * tiles, so one launch steps all of them. */

/* n consecutive kami_vbd_step(dt) calls.  The fused form runs steps_per_launch steps per launch with
 * the state kept on chip between them, and replays the launches from a CUDA graph (captured on the
 * first call for a given n).  body_transforms: host, 7 floats per step (rotation x y z w,
 * translation), or NULL to keep the current transform.  Asynchronous. */
kami_status kami_vbd_step_n(kami_vbd_handle h, float dt, int32_t n, const float* body_transforms, void* stream);

/* Tile shape: slots per lane C (even, >= the longest strand / 32; changing it moves the state to the
 * new tiles), warps per CTA (1, 2, 4, 8), steps per launch for kami_vbd_step_n (1..1024) and the
 * variant of the fused kernel (register_cap: 1 = plain; 120 = at most 120 registers, C = 2 only: 17
 * instead of 16 warps per SM; 168 = at most 168 registers, C = 4 only: 12 instead of 8 warps per SM;
 * 2 = packed FP32x2, C = 4 and colour2 only: each lane updates its two same-colour slots with one
 * paired instruction per operation; a cap for the other C runs the plain kernel).  0 leaves a value
 * unchanged. */
kami_status kami_vbd_set_tuning(kami_vbd_handle h, int32_t slots_per_lane, int32_t warps_per_block,
                                int32_t steps_per_launch, int32_t register_cap);
kami_status kami_vbd_get_tuning(kami_vbd_handle h, int32_t* slots_per_lane, int32_t* warps_per_block,
                                int32_t* steps_per_launch, int32_t* register_cap);

/* How the fused step's launches are scheduled (no counterpart in the reference).  0: one CTA per
 * warps_per_block tiles (or per group of tiles), placed on the SMs by the hardware.
 * KAMI_LAUNCH_PERSISTENT: at most as many CTAs as stay resident at once, each looping over every
 * gridDim-th unit of tiles; the results agree to the last bits (the kernels are compiled apart).
 * The autotuner times both and keeps the faster. */
enum { KAMI_LAUNCH_PERSISTENT = 1 };
kami_status kami_vbd_set_launch_mode(kami_vbd_handle h, int32_t mode);
kami_status kami_vbd_get_launch_mode(kami_vbd_handle h, int32_t* mode);

/* Times every tile shape on this handle's own strands (C in {min..4}, register cap {none, 120} for
 * C = 2, warps per CTA in {1,2,4,8}, steps per launch in {1,4,16}; trial_steps steps of dt each),
 * keeps the fastest and restores the simulation state and clock; the fastest shape is then timed
 * with each launch mode (kami_vbd_set_launch_mode) and keeps the fastest mode.
 * best = {C, warps, steps per launch, register cap}; best_rate in vertex-iters/s. */
kami_status kami_vbd_autotune(kami_vbd_handle h, float dt, int32_t trial_steps, int32_t best[4], double* best_rate);

/* ---- differentiable stepping ---------------------------------------------------------------------
 * No counterpart in the reference, which has no adjoint.  The fused colour2 step (wind, SDF and any
 * number of substeps) can record its iterates on a tape; kami_vbd_backward then runs the hand-written
 * adjoint of the recorded steps in reverse.  Typical use, checkpointing every k steps: restore a
 * checkpoint with kami_vbd_set_state, record the k steps of that segment, call kami_vbd_backward
 * with the adjoint of the segment's final state, and continue with the next earlier segment. */

/* Allocates a tape for up to max_steps recorded substeps of up to max_tiles warp tiles (0 = all tiles;
 * rounded up to whole groups of tiles) and the adjoint buffers (d loss / d qRest starts at zero); the
 * tile window starts as the first max_tiles tiles.  A tape substep costs (num_itr + 1) * 32 + 48 B
 * per slot.  KAMI_ERR_UNSUPPORTED for the sweep form or the Jacobi schedule. */
kami_status kami_vbd_tape_reserve(kami_vbd_handle h, int32_t max_steps, int64_t max_tiles);

/* Number of warp tiles of the device layout. */
kami_status kami_vbd_get_tile_count(kami_vbd_handle h, int64_t* num_tiles);

/* Tiles per group of the fused layout: 1 when every strand fits a tile, else the 2, 4 or 8 tiles that
 * a strand may run on across (no counterpart in the reference). */
kami_status kami_vbd_get_tiles_per_group(kami_vbd_handle h, int32_t* tiles_per_group);

/* Restricts recording and the adjoint to tiles [tile_begin, tile_end) (at most the tape's tiles; both
 * multiples of kami_vbd_get_tiles_per_group).  Strands never cross a group of tiles, so a large groom
 * is differentiated window by window: for each window, restore each checkpoint, record and run
 * kami_vbd_backward; the adjoint of vertices outside the window passes through unchanged. */
kami_status kami_vbd_set_tape_window(kami_vbd_handle h, int64_t tile_begin, int64_t tile_end);

/* kami_vbd_set_state for the strands of the tape window only (no counterpart in the reference): from
 * a whole-groom state buffer (kami_vbd_get_state layout) in device memory, restores the state of the
 * strands whose tiles lie in the window, and the step clock; the other strands keep their state.
 * Restoring a checkpoint window by window then moves 1/n of the state per window instead of all of
 * it.  With host memory, or a window that covers the whole groom, it is kami_vbd_set_state.  When the
 * window is smaller than the groom and the adjoints are in device memory, kami_vbd_backward likewise
 * reads and writes only the window's entries of the adjoint arrays.  The first such call on a layout
 * allocates a slot -> vertex map of 8 B per slot. */
kami_status kami_vbd_restore_tape_window(kami_vbd_handle h, const void* src, size_t bytes, int32_t memory);

/* kami_vbd_step that also records its iterates.  A step of ceil(dt / max_h) substeps takes as many
 * of the tape's max_steps entries (one per substep; KAMI_ERR_STATE when they do not fit). */
kami_status kami_vbd_step_record(kami_vbd_handle h, float dt, void* stream);

/* In: the adjoint (d loss / d state) of the state after the last recorded step, boundary order:
 * adj_x, adj_v, adj_vlast 3*V floats, adj_q 4*V floats.  Out (in place): the adjoint of the state
 * before the first recorded step.  Adds d loss / d qRest of the recorded steps to the accumulated
 * gradient and empties the tape.  Synchronous. */
kami_status kami_vbd_backward(kami_vbd_handle h, float* adj_x, float* adj_v, float* adj_vlast, float* adj_q,
                              int32_t memory, void* stream);

/* The accumulated d loss / d qRest (4*V floats, boundary order), and its reset to zero. */
kami_status kami_vbd_get_rest_darboux_grad(kami_vbd_handle h, float* xyzw, int32_t memory);
kami_status kami_vbd_zero_rest_darboux_grad(kami_vbd_handle h);

/* ---- one step without any device allocation ----------------------------------------------------
 * No counterpart in the reference (every reference path allocates through YarnBall::Sim).
 *
 * For callers that cannot let a library call cudaMalloc: an engine that owns all device memory
 * itself (a fixed pool or a hard memory budget), or a real-time frame loop where an allocation,
 * which can synchronise the whole device, would break the frame deadline.  Creating a handle
 * allocates, so such a caller keeps the solver state in its own device buffers, in boundary order,
 * and advances it with this entry point, which allocates nothing.
 *
 * It runs one KamiSimulator internal step like kami_vbd_step with the colour2 schedule and the sweep
 * kernels, but with no SDF pass and no finiteness check.  Scratch lives in a fixed __device__ array
 * for at most KAMI_NOALLOC_MAX_VERTICES vertices (12 MiB held by every device that loads the library
 * until exit); larger inputs are rejected with KAMI_ERR_UNSUPPORTED.  Every call made outside a
 * stream capture looks up that array's device address in the current context; a call made while
 * its stream captures reuses the address of the last such call on the device, so make the first
 * call on a device, and the first after a cudaDeviceReset, outside any capture.  All calls share
 * the scratch: calls whose work overlaps on the GPU race and must be serialised by the caller.
 * Per-vertex arrays hold what kami_vbd_create derives (inverse mass with pinned roots at 0, rest
 * length, stretch stiffness, orientations, stiffness-scaled rest Darboux quaternions).  The strand
 * offsets should satisfy strand_begin[0] == 0, strand_begin[num_strands] == num_vertices and be
 * increasing; they stay on the device and are not checked, but each strand is clamped to the
 * vertex range, so malformed offsets give wrong results, never an access out of bounds.  A dt
 * that is not finite, or that needs more than KAMI_MAX_SUBSTEPS substeps of max_h, is rejected. */
#define KAMI_NOALLOC_MAX_VERTICES 262144

typedef struct kami_vbd_noalloc_args {
    int64_t num_vertices;
    int32_t num_strands;
    const int32_t* strand_begin;    /* device, num_strands + 1 CSR offsets */
    float* positions;               /* device, 3 * V, updated in place */
    float* velocities;              /* device, 3 * V, updated in place */
    float* last_velocities;         /* device, 3 * V, updated in place (zero before the first call) */
    float* orientations;            /* device, 4 * V (x, y, z, w), updated in place */
    const float* rest_darboux;      /* device, 4 * V */
    const float* inv_mass;          /* device, V */
    const float* rest_length;       /* device, V */
    const float* stretch_stiffness; /* device, V */
    float clock[3];                 /* host: h of the previous call (max_h before the first), lastH, time */
} kami_vbd_noalloc_args;

/* settings: scalar fields of a kami_vbd_desc (gravity, damping, velocity_decay, acceleration_ratio,
 * external_force_multiplier, wind, num_itr, max_h, schedule); geometry fields are ignored, and a
 * non-NULL connection_index is KAMI_ERR_UNSUPPORTED.
 * Asynchronous on `stream` (a cudaStream_t; NULL = legacy default stream); args->clock is updated. */
kami_status kami_vbd_step_noalloc(const kami_vbd_desc* settings, kami_vbd_noalloc_args* args, float dt, void* stream);

/* Description of the last error on the calling thread ("" if none). */
const char* kami_vbd_last_error_string(void);

/* Library version string. */
const char* kami_vbd_version(void);

#ifdef __cplusplus
}
#endif

#endif /* KAMI_VBD_H_ */

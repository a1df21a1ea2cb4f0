/*
 * gg_step.h -- C ABI of the B200 GraGLeS2D level-set step.
 *
 * One context holds one grain network resident on one GPU: per-grain square
 * boxes (the reference's LSbox, src/box.h:68-111) with their distance
 * functions, IDLocal maps, comparison lists, contours, junctions and
 * neighbour characteristics.  The stage entry points are the stage methods
 * of the reference's time loop (grainhdl, src/grainhdl.h:115-141) and run
 * every grain of the network in one launch sequence on the device.
 *
 * Conventions
 *  - Grain IDs are the reference's: 1..N for grains, 0 for the domain
 *    boundary grain (src/grainhdl.h:153-160).
 *  - Every function returns 0 on success or a positive GG_E_* code; no
 *    C++ exception crosses this boundary.  gg_last_error() describes the
 *    last failure of a context.
 *  - Host arrays passed in are copied; the library owns all device memory.
 *  - A context is used from one host thread at a time.
 *  - Precision GG_PRECISION_PLAIN computes in FP64 and reproduces the
 *    reference's arithmetic; GG_PRECISION_BATCHED computes the bulk stages
 *    in FP32 (areas and energies still accumulate in FP64) and runs each
 *    step as one captured CUDA graph.
 */
#ifndef GG_STEP_H
#define GG_STEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GG_ABI_VERSION 1

enum {
    GG_OK = 0,
    GG_E_INVALID = 1,      /* bad argument or unsupported setting */
    GG_E_CUDA = 2,         /* CUDA runtime error */
    GG_E_IO = 3,           /* file missing or malformed */
    GG_E_STATE = 4,        /* call out of order (e.g. step before load) */
    GG_E_CAPACITY = 5,     /* a device arena, list or table overflowed */
    GG_E_NUMERIC = 6       /* a non-finite input value, or a NaN / infinity in a distance field or an area on
                              the device (GG_S_NAN) */
};

enum { GG_PRECISION_PLAIN = 0, GG_PRECISION_BATCHED = 1 };

/* Device status bits reported by gg_status(). */
enum {
    GG_S_ARENA_FULL = 1 << 0,
    GG_S_LIST_OVERFLOW = 1 << 1,
    GG_S_CONTOUR_OVERFLOW = 1 << 2,
    GG_S_JUNCTION_OVERFLOW = 1 << 3,
    GG_S_WALK_LIMIT = 1 << 4,
    GG_S_TABLE_RANGE = 1 << 5,
    GG_S_NEIGHBOUR_OVERFLOW = 1 << 6,
    GG_S_NAN = 1 << 7,
    GG_S_INDEX = 1 << 8,         /* an access the reference would have faulted on */
    GG_S_SECTOR_GUARD = 1 << 9,  /* a sector walk met a zero-length contour */
    GG_S_RETRY_LIMIT = 1 << 10   /* more than 64 contour re-extractions */
};

/*
 * Simulation settings used on the step path.  Field names follow the
 * parameters.xml tags parsed by Settings::initializeParameters
 * (src/Settings.cpp:111-283).  theta_ref_deg, gamma_hagb and m_hagb are
 * constants in the reference (src/box.cpp:1786-1787, 1846;
 * src/junction.cpp:40-41); they default to those constants.
 */
typedef struct gg_params {
    int32_t struct_size;              /* sizeof(gg_params) */
    int32_t precision;                /* GG_PRECISION_* */
    int32_t start_time;               /* StartTime */
    int32_t number_of_timesteps;      /* NumberOfTimesteps */
    int32_t analysis_timestep;        /* AnalysisTimestep */
    int32_t breakup_number;           /* BreakupNumber */
    int32_t number_of_particles;      /* NumberOfParticles */
    int32_t number_of_points_per_grain; /* NumberOfPointsPerGrain */
    int32_t domain_border_size;       /* DomainBorderSize */
    int32_t microstructure_gen_mode;  /* MicrostructureGenMode (0 and 4 supported) */
    int32_t convolution_mode;         /* ConvolutionMode (2 = Gaussian supported) */
    int32_t lattice_type;             /* LatticeType (0 = cubic supported) */
    int32_t is_isotropic_network;     /* IsIsotropicNetwork */
    int32_t use_mobility_model;       /* UseMobilityModel (0, 1) */
    int32_t identify_twins;           /* IdentifyTwins */
    int32_t research_mode;            /* ResearchMode (0 supported) */
    int32_t research_project;         /* ResearchProject */
    int32_t decouple_grains;          /* DecoupleGrains */
    int32_t grid_coarsement;          /* GridCoarsement (0, 1: gg_step and gg_convolution coarsen the grid when due) */
    int32_t use_stored_elastic_energy;/* UseStoredElasticEnergy (0, 1) */
    int32_t use_magnetic_field;       /* UseMagneticField (0, 1; parameters from the MagneticParams file) */
    int32_t discrete_sampling_rate;   /* DiscreteSamplingRate (bins of the MODF output) */
    /* control settings the step does not use; kept to be written back into
     * restart parameter files */
    int32_t plot_interval;            /* PlotInterval */
    int32_t use_texture;              /* UseTexture */
    int32_t execute_in_parallel;      /* ExecuteInParallel */
    int32_t maximum_number_of_threads;/* MaximumNumberOfThreads */
    int32_t neighbour_tracking;       /* NeighbourTracking */
    int32_t grain_scheduler;          /* GrainScheduler */
    /* library settings (no parameters.xml tag) */
    int32_t list_capacity;            /* comparison / second-order list entries per grain, 1..128 (0: 96);
                                         a longer list is a GG_E_CAPACITY error */
    int32_t reserved_i;
    double triple_point_drag;         /* TriplePointDrag */
    double constant_sector_radius;    /* ConstantSectorRadius (grid points) */
    double interpolating_sector_radius; /* InterpolatingSectorRadius (grid points) */
    double hagb_energy;               /* HAGB_Energy */
    double hagb_mobility;             /* HAGB_Mobility */
    double physical_domain_size;      /* Physical_Domain_Size */
    double time_slope;                /* GaussianKernelUserDefTimeSlope */
    double theta_ref_deg;             /* Read-Shockley cut-off angle */
    double gamma_hagb;                /* relative high-angle boundary energy */
    double m_hagb;                    /* relative high-angle boundary mobility */
    double dislocation_energy_per_m;  /* DislocEnPerM (scales the stored energies) */
    double box_default_stored_elastic_energy; /* BoxDefaultStoredElasticEnergy (domain boundary) */
    /* magnetic field: the tags of the file that MagneticParams names
     * (Settings::readMagneticFieldParams, src/Settings.cpp:291-347) */
    double vacuum_permeability;       /* VacuumPermeability */
    double magnetic_vector[3];        /* MagneticVector_x, _y, _z (unit field direction) */
    double delta_mag_sys;             /* deltaMagSys (susceptibility difference) */
    double magnetic_force_field;      /* MagneticForceField */
    double grid_coarsement_gradient;  /* GridCoarsementGradient */
    double arena_factor;              /* distance-field, spectrum and contour arenas hold this multiple (>= 1)
                                         of the initial network's totals (0: twice, and at least 2^20 values
                                         more); boxes outgrowing them stop the run with GG_E_CAPACITY */
    char read_from_filename[512];     /* ReadFromFilename (.bin ID field) */
    char additional_filename[512];    /* AdditionalFilename (.uds header) */
} gg_params;

/* Per-grain scalars, as reported by the reference's texture output
 * (TextureData, src/Structs.h; src/box.cpp:2296-2312). */
typedef struct gg_grain_stats {
    int32_t id;
    int32_t state;             /* 0 removed, 1 exists, 2 vanished this step */
    int32_t motion_regular;    /* LSbox::isMotionRegular */
    int32_t intersects_boundary;
    int32_t n_neighbours;      /* direct neighbours */
    int32_t contour_points;    /* contour length incl. closing point */
    int32_t box[4];            /* xmin, xmax, ymin, ymax of the current box */
    double area;               /* m_volume */
    double energy;             /* m_energy */
    double perimeter;          /* m_perimeter */
    double mean_da;            /* m_meanDa */
} gg_grain_stats;

typedef struct gg_ctx gg_ctx;

/* Fills defaults equal to Settings' static initialisers (src/Settings.cpp:26-79). */
int gg_params_default(gg_params* p);

/* Parses a parameters.xml (replaces Settings::initializeParameters,
 * src/Settings.cpp:84-289).  Unknown tags are ignored. */
int gg_params_from_xml(const char* path, gg_params* p);

/* Creates a context on a CUDA device (replaces grainhdl's constructor and
 * the settings part of grainhdl::setSimulationParameter,
 * src/grainhdl.cpp:56-136). */
int gg_create(const gg_params* p, int device, gg_ctx** out);
void gg_destroy(gg_ctx* ctx);
const char* gg_last_error(const gg_ctx* ctx);

/* Loads a voxelized microstructure (replaces grainhdl::read_HeaderCPG and
 * grainhdl::read_voxelized_microstructure, src/grainhdl.cpp:275-511).
 * ids: nn*nn int32 grain IDs, row-major, row outer; euler: 3 Bunge angles
 * per grain (index id-1); bbox: xmin, xmax, ymin, ymax, count per grain in
 * interior coordinates.  Grains with count 0 are absent, as in the reference. */
int gg_load_voxels(gg_ctx* ctx, int32_t nn, const int32_t* ids, int32_t n_grains, const double* euler,
                   const int32_t* bbox);
/* Same, reading the .uds/.bin pair named by the parameters (paths relative to
 * base_dir when not absolute). */
int gg_load_voxel_files(gg_ctx* ctx, const char* base_dir);
/* Stored elastic energies, one per grain (index id-1), the .uds storedEnergy
 * column that grainhdl::read_HeaderCPG reads when UseStoredElasticEnergy is
 * set (src/grainhdl.cpp:404-425); gg_load_voxel_files reads them from the
 * file.  Call after gg_load_voxels, before gg_distance_initialisation. */
int gg_load_stored_energy(gg_ctx* ctx, const double* stored, int32_t n_grains);

/* Loads grain contours, MicrostructureGenMode 0 (replaces
 * grainhdl::readMicrostructure, src/grainhdl.cpp:605-654, and the LSbox
 * read-from-file constructor, src/box.cpp:108-159).  Grain k (k = 1 ..
 * n_grains) is the k-th contour: offsets[k-1] .. offsets[k]-1 index its
 * points, xy[2p], xy[2p+1] in domain coordinates (clamped to [0, 1] as the
 * reference clamps them), and quat[4(k-1)] .. quat[4(k-1)+3] its
 * orientation quaternion, used as given.  A grain with no points is
 * absent; one with 1 or 2 points is refused.  The grid is
 * int(sqrt(NumberOfParticles) x NumberOfPointsPerGrain) points, as the
 * reference computes it for this mode (src/grainhdl.cpp:74-78). */
int gg_load_contours(gg_ctx* ctx, int32_t n_grains, const int32_t* offsets, const double* xy, const double* quat);
/* Same, reading the contour file ReadFromFilename names (a NETWORK_*.dat
 * restart file as gg_write_restart writes it; relative to base_dir when not
 * absolute).  Grains are numbered in file order, as the reference numbers
 * them; a record whose ID is at least the grain count raises the count to
 * that ID, and grains without a record are absent (the reference reads past
 * the end of the file there). */
int gg_load_contour_file(gg_ctx* ctx, const char* base_dir);

/* grainhdl::distanceInitialisation (src/grainhdl.cpp:728-753).  Mode-4 input
 * (src/box.cpp:322-341): +-h field, redistancing, contour.  Contour input
 * (src/box.cpp:342-400): the signed distance to the grain's polygon, clamped
 * to +-delta, sign from the crossing-number point-in-polygon test; the
 * contour stays the loaded polygon until the first level-set stage. */
int gg_distance_initialisation(gg_ctx* ctx);
/* grainhdl::find_neighbors (src/grainhdl.cpp:1258-1283): every grain whose box
 * intersects, in ascending ID order. */
int gg_find_neighbors(gg_ctx* ctx);
/* Replaces the initial comparison lists with caller-given ordered lists
 * (CSR over grains 1..N: offsets[N+1], ids); use to reproduce an exact
 * neighbour order (ties in the comparison take the first list member). */
int gg_set_neighbours(gg_ctx* ctx, const int32_t* offsets, const int32_t* ids);

/* Stage calls of one timestep, in the reference loop's order
 * (src/grainhdl.cpp:1049-1142); buffer switches are implicit.  `loop` is
 * the reference's loop counter (the corrector is off for loop 0). */
int gg_convolution(gg_ctx* ctx, int32_t loop);
int gg_update_second_order_neighbors(gg_ctx* ctx);
int gg_comparison(gg_ctx* ctx);
int gg_level_set(gg_ctx* ctx, int32_t loop);
int gg_redistancing(gg_ctx* ctx, int32_t loop);
/* grainhdl::get_biggestGrainVol: live-grain count and largest area. */
int gg_grain_count(gg_ctx* ctx, int32_t* current_nr_grains, double* max_volume);

/* Runs nsteps whole timesteps starting at loop index `loop`.  The batched
 * form replays one captured CUDA graph per step. */
int gg_step(gg_ctx* ctx, int32_t loop, int32_t nsteps);

/* Device status word (GG_S_* bits), accumulated since the last clear. */
int gg_status(gg_ctx* ctx, uint32_t* status, int32_t clear);

/* Per-grain scalars for grains 1..N (out has room for N entries). */
int gg_read_grain_stats(gg_ctx* ctx, gg_grain_stats* out, int32_t capacity);
/*
 * Parameter derivatives (no counterpart in the reference, which has no
 * derivative; the calibration interface the drop-in adds).  With tangents
 * enabled (before gg_distance_initialisation; plain form only), every step
 * also carries d phi / d p for p = (ThetaRefDegrees, HAGB_RelativeEnergy,
 * HAGB_RelativeMobility, TriplePointDrag): the tangent-linear step with the
 * step's discrete decisions fixed (comparison winners, contour edges,
 * redistancing candidates, corrector sectors).  gg_read_area_tangents
 * returns d area_g / d p of the contour of the last level set, 4 values per
 * grain for g = 1..N in that parameter order (theta per degree); capacity
 * counts doubles.  A loss gradient is sum_g dL/darea_g * out[4 (g-1) + k].
 */
int gg_tangent_enable(gg_ctx* ctx, int32_t enable);
int gg_read_area_tangents(gg_ctx* ctx, double* out, int32_t capacity);

/*
 * Analysis output of one timestep, the files grainhdl::save_Texture and
 * grainhdl::save_NrGrainsStats write (src/grainhdl.cpp:871-1023, 1225-1241),
 * in their formats, into `directory`:
 *  - Texture_<loop>.ori: per existing grain with regular motion, in ID order:
 *    ID, direct-neighbour count, boundary flag, area, mean dA / AnalysisTimestep,
 *    perimeter, energy, stored elastic energy, Bunge Euler angles;
 *  - MODF_<loop>.txt (anisotropic networks): the boundary-length-weighted
 *    misorientation distribution over DiscreteSamplingRate bins;
 *  - NrGrains&EnergyStatistics.txt: one line appended (the file is started
 *    afresh at loop 0): simulated time, grain count at the step's start,
 *    total boundary energy, grid size.
 * Call it after the step `loop` has completed (gg_step or gg_redistancing);
 * the reference calls it when (loop - StartTime) % AnalysisTimestep == 0 and
 * after the last step.  The simulated time is the sum of the reference's
 * per-step increments dt PhysicalDomainSize^2 / (TimeSlope HAGB_Energy
 * HAGB_Mobility) over the steps before `loop`.
 */
int gg_write_analysis(gg_ctx* ctx, const char* directory, int32_t loop);

/*
 * Restart files of one timestep, as grainhdl::save_Full_Microstructure_for_Restart
 * writes them (src/grainhdl.cpp:1179-1223, LSbox::plot_full_grain with
 * absolute coordinates, src/box.cpp:1552-1596), into `directory`:
 *  - NETWORK_NONAME_TIMESTEP_<loop>_GRAINS_<n>.dat: per existing grain, its ID,
 *    contour length and orientation quaternion, then its contour points in
 *    domain coordinates, then an empty line;
 *  - PARAMETERS_SIM_NONAME_TIMESTEP_<loop>_GRAINS_<n>.xml: the parameters
 *    (Settings::generateXMLParametersNode, src/Settings.cpp:363-400) with
 *    StartTime <loop>, NumberOfParticles <n>, MicrostructureGenMode 0 and the
 *    contour file as ReadFromFilename.
 * <n> is the grain count at the start of step `loop`, as for the statistics
 * file.  The reference writes them after step 0 of a voxelized input and after
 * step NumberOfTimesteps.  Call after step `loop` has completed.
 */
int gg_write_restart(gg_ctx* ctx, const char* directory, int32_t loop);

/* Number of grain slots N and the grid size (ngridpoints). */
int gg_dims(gg_ctx* ctx, int32_t* n_grains, int32_t* ngridpoints, double* h, double* delta, double* dt);

/* Writes the whole network state in the oracle dump format (one record). */
int gg_dump(gg_ctx* ctx, const char* path, int32_t steps_done, int32_t append);

/* Wall time of the device work of the last gg_step call, in milliseconds
 * (CUDA events on the context's stream). */
int gg_last_step_ms(gg_ctx* ctx, double* ms);

/* Sum over completed steps of the grains existing at each step's start
 * (the grain-updates behind grain-updates/s), counted on the device. */
int gg_grain_updates(gg_ctx* ctx, int64_t* updates);

/* Runs nsteps whole steps stage by stage with CUDA events between stages
 * and adds the device milliseconds of each stage to stage_ms[GG_NSTAGES]:
 * convolution, corrector, second-order lists, comparison, level set,
 * arena allocation, volume/energy/neighbours (in the batched form with the
 * next step's corrector sectors), redistancing, end of step
 * (the reference's stage timers, src/grainhdl.cpp:1146-1154). */
#define GG_NSTAGES 9
int gg_profile_steps(gg_ctx* ctx, int32_t loop, int32_t nsteps, double* stage_ms);

/* Algorithmic traffic model of the current network: sum of box areas of
 * existing grains, sum over grains of the overlap areas with their
 * comparison-list members, and the number of existing grains. */
int gg_traffic(gg_ctx* ctx, int64_t* sum_area, int64_t* sum_overlap, int32_t* n_exists);

/* Launch bins of the batched form, as gg_autotune chose them. */
typedef struct gg_tuning {
    int32_t compare_threads;  /* threads per CTA of the comparison */
    int32_t big_edge;         /* boxes with a larger edge go to the large-box redistancing kernel */
    int32_t conv_smem_edge;   /* the convolution keeps its intermediate in shared memory up to this edge */
    int32_t steps_run;        /* timesteps the sweep ran (the network advanced by them) */
    double ms_default;        /* device ms per step with the bins the context started with */
    double ms_tuned;          /* device ms per step with the chosen bins */
} gg_tuning;

/* Autotuner of the batched form's launch bins (no counterpart in the
 * reference, whose grain schedulers, src/SquaresGrainScheduler.cpp:24-147
 * and src/IterativeGrainScheduler.cpp:13-30, split grains among threads
 * statically).  Runs whole timesteps from `loop` as gg_step does, each
 * candidate for steps_per_candidate steps (0: 2), one knob at a time: the
 * large-box redistancing bin edge, the comparison's threads per CTA and the
 * convolution's shared-memory edge; a candidate is kept when it is more than
 * 1% faster.  No bin changes any result, so the steps it runs are ordinary
 * steps of the run.  The choice is kept for the context and, for the
 * process, for later contexts with the same largest box edge and grain
 * count.  The plain form returns at once (nothing to tune). */
int gg_autotune(gg_ctx* ctx, int32_t loop, int32_t steps_per_candidate, gg_tuning* out);

/* Kernels launched by gg_step's graph replays so far (batched form): the
 * kernel nodes of the captured step graph, counted when it is captured,
 * times the replays.  The plain form launches its stages from the host and
 * reports 0.  per_step (optional) receives the graph's kernel-node count. */
int gg_kernel_launches(gg_ctx* ctx, int64_t* total, int32_t* per_step);

/*
 * Allocation-free box convolution.  No counterpart in the reference: the
 * reference allocates its FFT scratch per thread.  For callers that cannot
 * allocate device memory (an application that passes this library buffers
 * from its own device memory pool and does not allow plug-ins to allocate),
 * this convolves one n x n box with the Gaussian kernel of the convolution
 * stage (src/box.cpp:622-695), with the plain form's arithmetic, so the
 * result is bit-identical to that stage.
 *  - d_in, d_out: caller-owned device buffers of n*n doubles, row-major.
 *  - dt, real_domain_size: the timestep and grid edge the kernel depends on.
 *  - stream: a cudaStream_t (NULL for the default stream); every call waits
 *    for that stream and returns after its work there has finished.
 * It calls no cudaMalloc, cudaFree or allocating library routine: its scratch
 * is a fixed array of about 300 KB compiled into the library, which every GPU
 * that loads the library holds until the process exits.  n must be in
 * 1..GG_STATIC_CONV_MAX_N, else GG_E_INVALID is returned.  No call can be
 * captured into a CUDA graph (each copies its tables from host memory and
 * waits for the stream): on a capturing stream it returns GG_E_INVALID and
 * issues nothing, so the capture stays valid.  All calls on a device share
 * the one scratch array, so calls that overlap on the GPU (from several host
 * threads or streams) race; serialise them.
 */
#define GG_STATIC_CONV_MAX_N 128
int gg_convolve_box_static(const double* d_in, double* d_out, int32_t n, double dt, int32_t real_domain_size,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GG_STEP_H */

# Builds the unmodified ParFlow CPU implementation from its own sources into
# oracle/_ref/ (test infrastructure: the reference arm of the benchmark and the
# pin for the C restatement in oracle/).  The reference's CMake build cannot be
# used here (its project() requires a Fortran compiler), so this recipe compiles
# the same source lists that pfsimulator/parflow_lib/CMakeLists.txt names,
# directly with gcc/g++.
#
#   make -f oracle/ref.mk -j8 REF=<parflow source tree>
#
# Products:
#   oracle/_ref/bin/parflow        AMPS "seq" layer, sequential loops
#   oracle/_ref/bin/parflow_omp    same, loops through the OpenMP backend
#                                  (pf_omploops.h), OMP_NUM_THREADS threads
#   oracle/_ref/bin/parflow_hook   seq build linked with oracle/ref_hooks.c via
#                                  ld --wrap: dumps F(p), J*v and PC(r) operands
#                                  when PFREF_DUMP_DIR is set.
#   oracle/_ref/bin/parflow_gpu    seq build with the GPU nonlinear-solver module
#                                  (parflow_b200/pfmodule/, libpfgpu.so) linked
#                                  in via ld --wrap; selected per run by
#                                  Solver.Nonlinear.GPU True (target gpu, after
#                                  libpfgpu.so is built).
# Nothing is written outside oracle/_ref/.  The two generated headers
# (parflow_config.h, pfversion.h) are written by this recipe from the values
# the CMake templates would substitute for a seq/no-hypre build.

ifeq ($(strip $(REF)),)
$(error REF is not set: make -f oracle/ref.mk REF=<parflow source tree>)
endif
HERE    := $(dir $(lastword $(MAKEFILE_LIST)))
OUT     := $(HERE)_ref
PL      := $(REF)/pfsimulator/parflow_lib
KS      := $(REF)/pfsimulator/kinsol
AM      := $(REF)/pfsimulator/amps
CJ      := $(REF)/pfsimulator/third_party/cjson
EXE     := $(REF)/pfsimulator/parflow_exe

CC      ?= gcc
CXX     ?= g++
# the OpenMP build needs a toolchain that ships libgomp's spec file
OMPCC   ?= $(if $(wildcard /usr/bin/gcc),/usr/bin/gcc,$(CC))
OMPCXX  ?= $(if $(wildcard /usr/bin/g++),/usr/bin/g++,$(CXX))
OPT     ?= -O2
INC     := -I$(OUT)/include -I$(AM)/seq -I$(AM)/common -I$(PL) -I$(KS) -I$(CJ)
CFLAGS  := $(OPT) -fcommon -w $(INC)

# pfsimulator/parflow_lib/CMakeLists.txt: SRC_FILES_CONST (Fortran advect.F /
# sadvect.F replaced by their shipped f2c translations *.win32.c)
CONST := advection_godunov bc_lb bc_pressure bc_pressure_package cghs char_vector \
  chebyshev comm_pkg communication computation compute_maximums compute_top_and_bottom \
  compute_patch_top compute_total_concentration constantRF constant_porosity create_grid \
  diag_scale diffuse_lb discretize_pressure distribute_usergrid dpofa dposl evaptranssum \
  gauinv general geom_t_solid geometry grgeom_list grgeom_octree grid hbt index_space \
  infinity_norm inputRF input_checks input_database input_porosity kinsol_nonlin_solver \
  kinsol_pc l2_error_norm line_process logging matdiag_scale max_field_value metadata \
  n_vector new_endpts nodiag_scale overlandsum pcg permeability_face perturb_lb pf_hypre \
  pf_n_vector pf_pfmg pf_pfmg_octree pf_smg pfield pgsRF ppcg printgrid printmatrix \
  printvector problem problem_bc_internal problem_bc_phase_saturation \
  problem_capillary_pressure problem_domain problem_dz_scale problem_eval problem_FBx \
  problem_FBy problem_FBz problem_geometries problem_ic_phase_concen problem_ic_phase_satur \
  problem_mannings problem_phase_heat_capacity problem_phase_internal_energy \
  problem_phase_mobility problem_phase_viscosity problem_porosity problem_real_space_z \
  problem_retardation problem_richards_bc_internal problem_saturation_constitutive \
  problem_spec_storage problem_thermal_conductivity problem_toposlope_x problem_toposlope_y \
  problem_wc_x problem_wc_y process_grid random ratqr read_parflow_binary \
  read_parflow_netcdf reg_from_stenc sadvection_godunov scale select_time_step \
  set_problem_data sim_shear solver solver_impes solver_lb solver_richards subsrf_sim \
  time_cycle_data timing total_velocity_face turning_bandsRF usergrid_input w_jacobi well \
  well_package wells_lb reservoir reservoir_package wrf_parflow cpl_parflow \
  write_clm_netcdf write_parflow_binary write_parflow_netcdf write_parflow_pdi \
  write_parflow_silo write_parflow_silo_pmpio advect.win32 sadvect.win32

# SRC_FILES_ARCH_TYPE_{0,1,2}: compiled as C for seq, as C++ + OpenMP for omp
ARCH0 := clustering grgeometry
ARCH1 := axpy copy innerprod matrix matvec mg_semi mg_semi_restrict mg_semi_prolong \
  nl_function_eval overlandflow_eval overlandflow_eval_diffusive overlandflow_eval_Kin \
  phase_velocity_face problem_phase_density problem_phase_rel_perm problem_phase_source \
  problem_saturation rb_GS_point richards_jacobian_eval seepage vector vector_utilities
ARCH2 := background calc_elevations globals pf_module problem_bc problem_bc_pressure \
  problem_ic_phase_pressure region
ARCH  := $(ARCH0) $(ARCH1) $(ARCH2)

KSSRC := iterativ kinsol kinspgmr llnlmath spgmr
AMSRC := amps_abort amps_clear amps_clock amps_exchange amps_ffopen amps_find_powers \
  amps_fopen amps_invoice amps_io amps_newhandle amps_newpackage amps_print amps_sfbcast \
  amps_sfclose amps_sfopen amps_wait signal

SEQ_OBJ := $(addprefix $(OUT)/seq/pl_,$(addsuffix .o,$(CONST) $(ARCH))) \
           $(addprefix $(OUT)/seq/ks_,$(addsuffix .o,$(KSSRC))) \
           $(addprefix $(OUT)/seq/am_,$(addsuffix .o,$(AMSRC))) \
           $(OUT)/seq/cjson.o $(OUT)/seq/dsign.o
OMP_OBJ := $(addprefix $(OUT)/omp/pl_,$(addsuffix .o,$(CONST))) \
           $(addprefix $(OUT)/omp/a0_,$(addsuffix .o,$(ARCH0))) \
           $(addprefix $(OUT)/omp/a1_,$(addsuffix .o,$(ARCH1))) \
           $(addprefix $(OUT)/omp/a2_,$(addsuffix .o,$(ARCH2))) \
           $(addprefix $(OUT)/omp/ks_,$(addsuffix .o,$(KSSRC))) \
           $(addprefix $(OUT)/omp/am_,$(addsuffix .o,$(AMSRC))) \
           $(OUT)/omp/cjson.o $(OUT)/seq/dsign.o

WRAPS := -Wl,--wrap=KINSolFunctionEval -Wl,--wrap=KINSolMatVec -Wl,--wrap=KinsolPC \
         -Wl,--wrap=RichardsJacobianEval

GPU_LIBDIR := $(abspath $(HERE)../parflow_b200)
GPU_WRAPS := $(foreach f,KinsolNonlinSolver KinsolNonlinSolverInitInstanceXtra \
               KinsolNonlinSolverFreeInstanceXtra KinsolNonlinSolverNewPublicXtra \
               KinsolNonlinSolverFreePublicXtra KinsolNonlinSolverSizeOfTempData,-Wl,--wrap=$(f))

all: $(OUT)/bin/parflow $(OUT)/bin/parflow_omp $(OUT)/bin/parflow_hook $(OUT)/bin/parflow_gpu

seq: $(OUT)/bin/parflow $(OUT)/bin/parflow_hook

gpu: $(OUT)/bin/parflow_gpu

HDRS := $(OUT)/include/parflow_config.h $(OUT)/include/pfversion.h

$(OUT)/include/parflow_config.h:
	@mkdir -p $(dir $@)
	@printf '%s\n' '#ifndef PARFLOW_CONFIG_H' '#define PARFLOW_CONFIG_H' \
	  '#define PARFLOW_AMPS_LAYER' '#define AMPS' \
	  '#define PARFLOW_HAVE_GETTIMEOFDAY' '#define CASC_HAVE_GETTIMEOFDAY' \
	  '#define PARFLOW_ENABLE_TIMING' '#define PF_TIMING' \
	  '#define PARFLOW_HAVE_MALLOC_H' '#define HAVE_MALLOC_H' \
	  '#define PARFLOW_HAVE_MALLINFO2' \
	  '#define PARFLOW_HYPRE_VERSION_MAJOR 0' '#define PARFLOW_HYPRE_VERSION_MINOR 0' \
	  '#define PARFLOW_HYPRE_VERSION_PATCH 0' '#endif' > $@

$(OUT)/include/pfversion.h:
	@mkdir -p $(dir $@)
	@printf '%s\n' '#ifndef PARFLOW_VERSION_H' '#define PARFLOW_VERSION_H' \
	  '#define PARFLOW_VERSION_STRING "3.15.0"' '#define PARFLOW_VERSION "3.15.0"' \
	  '#define PARFLOW_VERSION_MAJOR 3' '#define PARFLOW_VERSION_MINOR 15' \
	  '#define PARFLOW_VERSION_PATCH 0' '#define PARFLOW_VERSION_HASH ""' \
	  '#define PARFLOW_VERSION_EXTRA ""' '#endif' > $@

# ---- seq ------------------------------------------------------------------
$(OUT)/seq/pl_%.o: $(PL)/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@
$(OUT)/seq/ks_%.o: $(KS)/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@
$(OUT)/seq/am_%.o: $(AM)/common/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@
$(OUT)/seq/cjson.o: $(CJ)/cJSON.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@
$(OUT)/seq/main.o: $(EXE)/main.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@
$(OUT)/seq/dsign.o: $(HERE)ref_dsign.c
	@mkdir -p $(dir $@)
	$(CC) $(OPT) -c $< -o $@
$(OUT)/seq/hooks.o: $(HERE)ref_hooks.c $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/bin/parflow: $(SEQ_OBJ) $(OUT)/seq/main.o
	@mkdir -p $(dir $@)
	$(CC) -o $@ $^ -lm

$(OUT)/bin/parflow_hook: $(SEQ_OBJ) $(OUT)/seq/main.o $(OUT)/seq/hooks.o
	@mkdir -p $(dir $@)
	$(CC) -o $@ $^ $(WRAPS) -lm

# the GPU module against the reference's headers; libpfgpu.so is found next
# to the package at run time (rpath relative to the binary)
$(OUT)/seq/kinsol_gpu.o: $(HERE)../parflow_b200/pfmodule/kinsol_gpu_nonlin_solver.c \
                         $(HERE)../include/pfgpu.h $(HDRS)
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -I$(HERE)../include -c $< -o $@

$(OUT)/bin/parflow_gpu: $(SEQ_OBJ) $(OUT)/seq/main.o $(OUT)/seq/kinsol_gpu.o \
                        $(GPU_LIBDIR)/libpfgpu.so
	@mkdir -p $(dir $@)
	$(CC) -o $@ $(SEQ_OBJ) $(OUT)/seq/main.o $(OUT)/seq/kinsol_gpu.o $(GPU_WRAPS) \
	  -L$(GPU_LIBDIR) -lpfgpu -Wl,-rpath,'$$ORIGIN/../../../parflow_b200' -lstdc++ -lm

# ---- OpenMP -----------------------------------------------------------------
OMPDEF := -DPARFLOW_HAVE_OMP -fopenmp
$(OUT)/omp/pl_%.o: $(PL)/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCC) $(CFLAGS) $(OMPDEF) -c $< -o $@
$(OUT)/omp/a0_%.o: $(PL)/%.cpp $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCXX) $(CFLAGS) $(OMPDEF) -DPF_COMP_UNIT_TYPE=0 -c $< -o $@
$(OUT)/omp/a1_%.o: $(PL)/%.cpp $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCXX) $(CFLAGS) $(OMPDEF) -DPF_COMP_UNIT_TYPE=1 -c $< -o $@
$(OUT)/omp/a2_%.o: $(PL)/%.cpp $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCXX) $(CFLAGS) $(OMPDEF) -DPF_COMP_UNIT_TYPE=2 -c $< -o $@
$(OUT)/omp/ks_%.o: $(KS)/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCC) $(CFLAGS) $(OMPDEF) -c $< -o $@
$(OUT)/omp/am_%.o: $(AM)/common/%.c $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCC) $(CFLAGS) $(OMPDEF) -c $< -o $@
$(OUT)/omp/cjson.o: $(CJ)/cJSON.c $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCC) $(CFLAGS) -c $< -o $@
$(OUT)/omp/main.o: $(EXE)/main.c $(HDRS)
	@mkdir -p $(dir $@)
	$(OMPCC) $(CFLAGS) $(OMPDEF) -c $< -o $@

$(OUT)/bin/parflow_omp: $(OMP_OBJ) $(OUT)/omp/main.o
	@mkdir -p $(dir $@)
	$(OMPCXX) -fopenmp -o $@ $^ -lm

.PHONY: all seq gpu

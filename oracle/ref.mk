# Test infrastructure: builds the reference SKIRT 9 CPU code from its own sources into
# oracle/_ref/ with a plain Makefile (the reference's CMake project is not used).
#
#   make -f oracle/ref.mk -j8            # from the repository root
#
# Products (all under oracle/_ref/, git-ignored):
#   lib/lib*.a                      the reference libraries (SMILE + SKIRT core/utils/...)
#   exe/skirt/bin/skirt             the reference command-line program (CPU path, `-t N`)
#   exe/skirt/bin/skirt_export      harness: loads a ski file through the reference's own
#                                   SimulationItem tree and exports grids, medium state,
#                                   mix tables and reference path segments as .npy files
#   git/SKIRT/resources/            placeholder so FilePaths (SKIRT/core/FilePaths.cpp:33)
#                                   finds its built-in resource directory relative to the
#                                   executable (../../../git/SKIRT/resources)
#
# The only configure-time inputs of the reference build are SMILE/build/version_in.h and a
# timestamp header; this recipe writes its own two-line stand-ins for both. Nothing on the
# photon-packet path reads them.

REF     ?= /root/reference
HERE    := $(patsubst %/,%,$(dir $(lastword $(MAKEFILE_LIST))))
OUT     := $(HERE)/_ref
OBJ     := $(OUT)/obj
LIB     := $(OUT)/lib
GEN     := $(OUT)/gen
BIN     := $(OUT)/exe/skirt/bin
RES     := $(OUT)/git/SKIRT/resources

CXX     ?= g++
CC      ?= gcc
# Release flags of the reference (CMake Release default for GNU): -O3 -DNDEBUG, C++14.
CXXFLAGS_REF := -O3 -DNDEBUG -std=c++14 -w -pthread
CFLAGS_REF   := -O3 -DNDEBUG -w -DFF_NO_UNISTD_H=1

S_FUND  := $(REF)/SMILE/fundamentals
S_SCH   := $(REF)/SMILE/schema
S_SER   := $(REF)/SMILE/serialize
S_BLD   := $(REF)/SMILE/build
K_CORE  := $(REF)/SKIRT/core
K_UTIL  := $(REF)/SKIRT/utils
K_MPI   := $(REF)/SKIRT/mpi
K_FITS  := $(REF)/SKIRT/fitsio
K_VORO  := $(REF)/SKIRT/voro
K_TET   := $(REF)/SKIRT/tetgen
K_MAIN  := $(REF)/SKIRT/main

INC_CORE := -I$(S_SCH) -I$(S_FUND) -I$(K_FITS) -I$(K_VORO) -I$(K_MPI) -I$(K_UTIL) -isystem $(K_TET)
INC_MAIN := -I$(S_SER) -I$(S_SCH) -I$(S_FUND) -I$(S_BLD) -I$(GEN) -I$(K_CORE) -I$(K_MPI) -I$(K_UTIL)

define objs_of
$(patsubst $(1)/%,$(OBJ)/$(2)/%.o,$(wildcard $(1)/*.$(3)))
endef

O_FUND := $(call objs_of,$(S_FUND),fundamentals,cpp)
O_SCH  := $(call objs_of,$(S_SCH),schema,cpp)
O_SER  := $(call objs_of,$(S_SER),serialize,cpp)
O_BLD  := $(OBJ)/build/BuildInfo.cpp.o
O_CORE := $(call objs_of,$(K_CORE),skirtcore,cpp)
O_UTIL := $(call objs_of,$(K_UTIL),utils,cpp)
O_MPI  := $(call objs_of,$(K_MPI),mpi,cpp)
O_FITS := $(call objs_of,$(K_FITS),fitsio,c)
O_VORO := $(call objs_of,$(K_VORO),voro,cc)
O_TET  := $(call objs_of,$(K_TET),tetgen,cxx)
O_MAIN := $(call objs_of,$(K_MAIN),main,cpp)
O_MAINLIB := $(OBJ)/main/SkirtCommandLineHandler.cpp.o

LIBS := $(LIB)/libserialize.a $(LIB)/libschema.a $(LIB)/libfundamentals.a $(LIB)/libbuild.a \
        $(LIB)/libskirtcore.a $(LIB)/libfitsio.a $(LIB)/libvoro.a $(LIB)/libmpi.a $(LIB)/libutils.a \
        $(LIB)/libtetgen.a
LINK_LIBS := -Wl,--start-group $(LIBS) -Wl,--end-group -pthread -ldl

all: $(BIN)/skirt $(BIN)/skirt_export $(RES)/placeholder.txt $(BIN)/skirt_gpu $(BIN)/skirt_oracle $(BIN)/skirt_refgpu

$(RES)/placeholder.txt:
	@mkdir -p $(RES)
	@echo "built-in resource directory marker for the reference build in oracle/_ref" > $@

$(GEN)/version.h:
	@mkdir -p $(GEN)
	@printf '#ifndef VERSION_HPP\n#define VERSION_HPP\n#define PROJECT_VERSION "v9.0"\n#endif\n' > $@

$(GEN)/timestamp.h:
	@mkdir -p $(GEN)
	@printf '#ifndef TIMESTAMP_H\n#define TIMESTAMP_H\n#define BUILD_DATE "oracle"\n#define BUILD_TIME "oracle"\n#define COMMIT_HASH "reference"\n#endif\n' > $@

$(OBJ)/fundamentals/%.o: $(S_FUND)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_FUND) -c $< -o $@
$(OBJ)/schema/%.o: $(S_SCH)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_FUND) -c $< -o $@
$(OBJ)/serialize/%.o: $(S_SER)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_SCH) -I$(S_FUND) -c $< -o $@
$(OBJ)/build/%.o: $(S_BLD)/% $(GEN)/version.h $(GEN)/timestamp.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_FUND) -I$(GEN) -c $< -o $@
$(OBJ)/skirtcore/%.o: $(K_CORE)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_CORE) -c $< -o $@
# AdaptiveMeshSnapshot::Node::appendTraversalData (AdaptiveMeshSnapshot.cpp:193-198) assigns
# `childIndex[begin + l] = <recursive call that grows childIndex>`; C++14 leaves the two operands
# unsequenced and GCC takes the element address first, so the write can land in the freed buffer
# (heap corruption, or traversal arrays with -1 entries). C++17 evaluates the right operand first:
# this one file is compiled as C++17, which changes nothing else.
$(OBJ)/skirtcore/AdaptiveMeshSnapshot.cpp.o: $(K_CORE)/AdaptiveMeshSnapshot.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -std=c++17 $(INC_CORE) -c $< -o $@
$(OBJ)/utils/%.o: $(K_UTIL)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_FUND) -c $< -o $@
$(OBJ)/mpi/%.o: $(K_MPI)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -I$(S_FUND) -c $< -o $@
$(OBJ)/fitsio/%.o: $(K_FITS)/%
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS_REF) -c $< -o $@
$(OBJ)/voro/%.o: $(K_VORO)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -c $< -o $@
$(OBJ)/tetgen/%.o: $(K_TET)/%
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) -DTETLIBRARY -c $< -o $@
$(OBJ)/main/%.o: $(K_MAIN)/% $(GEN)/version.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_MAIN) -c $< -o $@

$(LIB)/libfundamentals.a: $(O_FUND)
$(LIB)/libschema.a: $(O_SCH)
$(LIB)/libserialize.a: $(O_SER)
$(LIB)/libbuild.a: $(O_BLD)
$(LIB)/libskirtcore.a: $(O_CORE)
$(LIB)/libutils.a: $(O_UTIL)
$(LIB)/libmpi.a: $(O_MPI)
$(LIB)/libfitsio.a: $(O_FITS)
$(LIB)/libvoro.a: $(O_VORO)
$(LIB)/libtetgen.a: $(O_TET)
$(LIB)/%.a:
	@mkdir -p $(LIB)
	@rm -f $@
	ar rcs $@ $^

$(BIN)/skirt: $(O_MAIN) $(LIBS)
	@mkdir -p $(BIN)
	$(CXX) -o $@ $(O_MAIN) $(LINK_LIBS)

# the export harness: reference libraries + the command-line handler object + our harness TU
$(OBJ)/harness/skirt_export.o: $(HERE)/harness/skirt_export.cpp $(GEN)/version.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_MAIN) $(INC_CORE) -c $< -o $@

$(BIN)/skirt_export: $(OBJ)/harness/skirt_export.o $(O_MAINLIB) $(LIBS)
	@mkdir -p $(BIN)
	$(CXX) -o $@ $(OBJ)/harness/skirt_export.o $(O_MAINLIB) $(LINK_LIBS)

# The bridged program: the reference's skirt with the life-cycle hooks (patch_hooks.py, applied to
# copies under $(OUT)/patched/) and the SKIRT-side bridge of the B200 library
# (skirt9-gpu_b200/bridge/SkgpuLifeCycle.cpp), linked against lib/libskgpu.so. `skirt_gpu -g run.ski`
# runs the ski file's life-cycle segments on the B200; without -g it is the reference program.
PKG     := $(HERE)/../skirt9-gpu_b200
BRIDGE  := $(PKG)/bridge
PATCHED := $(OUT)/patched
O_BRIDGE := $(OBJ)/bridge/MonteCarloSimulation.o $(OBJ)/bridge/SkirtCommandLineHandler.o $(OBJ)/bridge/SkgpuLifeCycle.o

$(PATCHED)/MonteCarloSimulation.cpp $(PATCHED)/SkirtCommandLineHandler.cpp: $(HERE)/patch_hooks.py $(K_CORE)/MonteCarloSimulation.cpp $(K_MAIN)/SkirtCommandLineHandler.cpp
	python3 $(HERE)/patch_hooks.py $(REF) $(PATCHED)

$(OBJ)/bridge/MonteCarloSimulation.o: $(PATCHED)/MonteCarloSimulation.cpp $(BRIDGE)/SkgpuLifeCycle.hpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_CORE) -I$(K_CORE) -I$(BRIDGE) -c $< -o $@
$(OBJ)/bridge/SkirtCommandLineHandler.o: $(PATCHED)/SkirtCommandLineHandler.cpp $(BRIDGE)/SkgpuLifeCycle.hpp $(GEN)/version.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_MAIN) -I$(K_MAIN) -I$(BRIDGE) -c $< -o $@
$(OBJ)/bridge/SkgpuLifeCycle.o: $(BRIDGE)/SkgpuLifeCycle.cpp $(BRIDGE)/SkgpuLifeCycle.hpp $(HERE)/../include/skgpu.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_MAIN) $(INC_CORE) -I$(BRIDGE) -I$(HERE)/../include -c $< -o $@

$(BIN)/skirt_gpu: $(O_BRIDGE) $(filter-out $(O_MAINLIB),$(O_MAIN)) $(LIBS) $(PKG)/lib/libskgpu.so
	@mkdir -p $(BIN)
	$(CXX) -o $@ $(O_BRIDGE) $(filter-out $(O_MAINLIB),$(O_MAIN)) $(LINK_LIBS) -L$(PKG)/lib -lskgpu \
	    -Wl,-rpath,'$$ORIGIN/../../../../../skirt9-gpu_b200/lib'

bridge: $(BIN)/skirt_gpu

# The reference's own GPU route for a second baseline: the unmodified reference program except for
# a copy of GpuAcceleration.cpp whose driver-symbol loader prefers the versioned entry points
# (patch_refgpu.py; on this pool's driver the original resolves the legacy cuCtxCreate and its GPU
# runtime does not start). `skirt_refgpu -g run.ski` runs the reference's GPU layer.
$(PATCHED)/GpuAcceleration.cpp: $(HERE)/patch_refgpu.py $(K_CORE)/GpuAcceleration.cpp
	python3 $(HERE)/patch_refgpu.py $(REF) $(PATCHED)
$(OBJ)/refgpu/GpuAcceleration.o: $(PATCHED)/GpuAcceleration.cpp
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_CORE) -I$(K_CORE) -c $< -o $@
$(BIN)/skirt_refgpu: $(OBJ)/refgpu/GpuAcceleration.o $(O_MAIN) $(LIBS)
	@mkdir -p $(BIN)
	$(CXX) -o $@ $(OBJ)/refgpu/GpuAcceleration.o $(O_MAIN) $(LINK_LIBS)

refgpu: $(BIN)/skirt_refgpu

# Test infrastructure: the same bridged program with the bridge's skgpu_* calls renamed to the CPU
# oracle's or_* entry points (same signatures, oracle/skoracle.h), linked against
# oracle/_build/liboracle.so: runs the bridge's flattening and fetch logic end to end without a GPU
# (tests/test_bridge_cpu.py).
BRIDGE_FNS := create destroy last_error abi_version device_count upload_grid_cartesian upload_grid_sphere1d \
    upload_grid_octree upload_medium upload_dust_mix upload_rf_grid upload_instruments upload_sources set_options \
    clear_tallies run_primary fetch_instrument fetch_instrument_components fetch_radiation_field \
    upload_dust_emission upload_radiation_field prepare_secondary run_secondary \
    set_instrument_scattering_levels set_instrument_bands fetch_instrument_levels \
    upload_grid_sphere2d upload_grid_sphere3d upload_grid_cylinder2d upload_grid_cylinder3d \
    upload_grid_adaptive_mesh upload_grid_voronoi upload_grid_tetra upload_voronoi_cell_boxes \
    set_instrument_observer
BRIDGE_ORACLE_DEFS := $(foreach f,$(BRIDGE_FNS),-Dskgpu_$(f)=or_$(f)) -Dskgpu_ctx=or_ctx -include $(HERE)/skoracle.h

$(OBJ)/bridge/SkgpuLifeCycle_oracle.o: $(BRIDGE)/SkgpuLifeCycle.cpp $(BRIDGE)/SkgpuLifeCycle.hpp $(HERE)/skoracle.h
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS_REF) $(INC_MAIN) $(INC_CORE) -I$(BRIDGE) -I$(HERE)/../include $(BRIDGE_ORACLE_DEFS) -c $< -o $@

$(BIN)/skirt_oracle: $(OBJ)/bridge/MonteCarloSimulation.o $(OBJ)/bridge/SkirtCommandLineHandler.o \
                     $(OBJ)/bridge/SkgpuLifeCycle_oracle.o $(filter-out $(O_MAINLIB),$(O_MAIN)) $(LIBS) $(HERE)/_build/liboracle.so
	@mkdir -p $(BIN)
	$(CXX) -o $@ $(OBJ)/bridge/MonteCarloSimulation.o $(OBJ)/bridge/SkirtCommandLineHandler.o \
	    $(OBJ)/bridge/SkgpuLifeCycle_oracle.o $(filter-out $(O_MAINLIB),$(O_MAIN)) $(LINK_LIBS) \
	    -L$(HERE)/_build -loracle -Wl,-rpath,'$$ORIGIN/../../../../_build'

.PHONY: all bridge refgpu

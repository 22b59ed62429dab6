# Builds the reference's own MPM path (PhysBAM Public_Library, read in place)
# into oracle/_ref/ so that tests can pin the CPU restatement against it.
# Test infrastructure only: nothing in the product links or loads this.
#
#   make -f oracle/ref.mk -j8 REF=<PhysBAM checkout>
#
# Only the library layers the explicit MPM driver links against are compiled.
# Four sources are skipped: they need boost or cblas, which are absent, or do
# not compile with g++ 13 (a pointer comparison); none is on the MPM path.
REF ?= $(PHYSBAM_REFERENCE)
$(if $(REF),,$(error set REF (or PHYSBAM_REFERENCE) to the PhysBAM checkout))
OUT ?= $(dir $(lastword $(MAKEFILE_LIST)))_ref
PL  := $(REF)/Public_Library
LAYERS := Core Tools Grid_Tools Grid_PDE Geometry Rigids Deformables Solids Hybrid_Methods
SKIP := $(PL)/Geometry/Images/HIDDEN_SURFACE_PRIMITIVES.cpp \
        $(PL)/Hybrid_Methods/Examples_And_Drivers/MPM_MAC_DRIVER.cpp \
        $(PL)/Solids/Meshing/RED_GREEN_TRIANGLES.cpp \
        $(PL)/Solids/Meshing/RED_GREEN_TETRAHEDRA.cpp
SRCS := $(filter-out $(SKIP),$(foreach L,$(LAYERS),$(shell find $(PL)/$(L) -name '*.cpp')))
OBJS := $(patsubst $(PL)/%.cpp,$(OUT)/obj/%.o,$(SRCS))
CXX := g++
CXXFLAGS := -std=gnu++14 -O2 -fPIC -fopenmp -DUSE_OPENMP -DNDEBUG -fno-math-errno \
            -fno-signed-zeros -include limits -include functional -fpermissive -w -I$(PL)

HERE := $(dir $(lastword $(MAKEFILE_LIST)))
MPM_LIB := $(HERE)../physbam_b200/libphysbam_mpm.so

all: $(OUT)/libphysbam_ref.so $(OUT)/ref_scene $(OUT)/ref_b200

$(OUT)/obj/%.o: $(PL)/%.cpp
	@mkdir -p $(dir $@)
	@$(CXX) $(CXXFLAGS) -c $< -o $@

$(OUT)/libphysbam_ref.so: $(OBJS)
	$(CXX) -shared -fopenmp -o $@ $^ -lz

$(OUT)/ref_scene: $(HERE)ref_scene.cpp $(HERE)ref_scene.h $(OUT)/libphysbam_ref.so
	$(CXX) $(CXXFLAGS) -o $@ $< -L$(OUT) -lphysbam_ref -Wl,-rpath,'$$ORIGIN' -Wl,--allow-shlib-undefined -lz

# the reference-side binding (include/mpm_physbam.hpp) driving MPM_EXAMPLE scenes on the GPU
$(OUT)/ref_b200: $(HERE)ref_b200.cpp $(HERE)ref_scene.h $(HERE)../include/mpm_physbam.hpp $(OUT)/libphysbam_ref.so $(MPM_LIB)
	$(CXX) $(CXXFLAGS) -I$(HERE)../include -o $@ $< -L$(OUT) -lphysbam_ref -L$(dir $(MPM_LIB)) -lphysbam_mpm \
	    -Wl,-rpath,'$$ORIGIN' -Wl,-rpath,'$$ORIGIN/../../physbam_b200' -Wl,--allow-shlib-undefined -lz

.PHONY: all

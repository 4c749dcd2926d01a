# Builds oracle/_ref/libref.so: the reference's own sources compiled where
# they lie under /root/reference (read-only), plus oracle/ref_harness.cu.
# Also oracle/_ref/libdropin.so: the drop-in results_with_given_normal of
# tests/dropin/ compiled against the reference's headers and linked with
# libref.so and this repository's libqmcrt.so (when that is built).
# Test infrastructure only; outputs go to oracle/_ref/ (git-ignored).
#
# Portability shims, all in _ref/shim (generated, never edited sources):
#  - compact_sample.cuh includes <thrust\device_ptr.h> etc. with Windows
#    backslashes; files with those literal names forward to <thrust/...>,
#    and add <thrust/device_malloc.h>, which compact_sample.cu uses without
#    including it.
#  - -Xcompiler -fpermissive accepts the extra qualification at
#    heliostat.cuh:59-60; -diag-suppress silences nvcc's warnings for
#    `const T const` (global_function.cuh:123-124) and friends.
# scene_file_proc.cpp and solar_scene.cpp are not built: scene_file_proc.h
# declares an enumerator `norm` that collides with CUDA's norm(); the harness
# builds scenes from the reference classes directly instead.
REF ?= /root/reference/Hu_smooth/ClassedSunRay
OUT := _ref
NVCC ?= /usr/local/cuda/bin/nvcc
FLAGS := -O2 -gencode arch=compute_100a,code=sm_100a -Xcompiler -fPIC -Xcompiler -fpermissive -w \
         -diag-suppress 83,940,177,550 -I$(OUT)/shim -I$(REF)
SRCS_CU := scene_instance_process.cu random_generator.cu steps_for_raytracing.cu poisson_disk.cu \
           compact_sample.cu rectgrid_raytracing.cu ray_tracing.cu image_smooth.cu
SRCS_CPP := scene_instance_process.cpp random_generator.cpp common_var.cpp heliostat.cpp grid.cpp receiver.cpp \
            recthelio_tracing.cpp image_save.cpp
OBJS := $(addprefix $(OUT)/obj/,$(SRCS_CU:.cu=.cu.o) $(SRCS_CPP:.cpp=.cpp.o))
SHIMS := device_ptr copy host_vector device_vector

DROPIN := ../tests/dropin
LIBQMCRT := ../onemirror_b200/lib/libqmcrt.so
DROPIN_LIB := $(if $(wildcard $(LIBQMCRT)),$(OUT)/libdropin.so)

all: $(OUT)/libref.so $(DROPIN_LIB)

$(OUT)/shim/.done:
	mkdir -p $(OUT)/shim $(OUT)/obj
	for f in $(SHIMS); do printf '#include <thrust/%s.h>\n#include <thrust/device_malloc.h>\n' $$f > "$(OUT)/shim/thrust\\$$f.h"; done
	touch $@

$(OUT)/obj/%.cu.o: $(REF)/%.cu $(OUT)/shim/.done
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/obj/%.cpp.o: $(REF)/%.cpp $(OUT)/shim/.done
	$(NVCC) $(FLAGS) -x cu -c $< -o $@

$(OUT)/obj/ref_harness.o: ref_harness.cu $(OUT)/shim/.done
	$(NVCC) $(FLAGS) -c $< -o $@

$(OUT)/libref.so: $(OBJS) $(OUT)/obj/ref_harness.o
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $^ -lcurand

$(OUT)/obj/dropin_%.o: $(DROPIN)/%.cu $(OUT)/shim/.done ../include/qmcrt.h
	$(NVCC) $(FLAGS) -I../include -c $< -o $@

$(OUT)/libdropin.so: $(OUT)/obj/dropin_results_with_given_normal.o $(OUT)/obj/dropin_harness.o $(OUT)/libref.so $(LIBQMCRT)
	$(NVCC) -shared -gencode arch=compute_100a,code=sm_100a -o $@ $(filter %.o,$^) -L$(OUT) -lref \
	    -L../onemirror_b200/lib -lqmcrt -Xlinker -rpath,'$$ORIGIN' -Xlinker -rpath,'$$ORIGIN/../../onemirror_b200/lib'

clean:
	rm -rf $(OUT)

.PHONY: all clean

# Builds the reference implementation's own CPU path (tags::CPU, tags::CPU::SSE,
# tags::CPU::MultiCore::SSE) from the reference sources where they lie, plus the
# driver programs in this directory that call it.  Outputs go to oracle/_ref/ only.
#
#   make -f oracle/ref.mk REF=<reference checkout> -j8   (or HONEI_REFERENCE=<checkout>)
#
# The reference is gnu++98 code; -fpermissive silences its pre-C++11 idioms and
# -std=gnu++98 is required (C++11 makes `bind` ambiguous in util/log.cc and
# util/time_stamp.hh uses GNU `typeof`).  -march=x86-64-v3 (AVX2/FMA) instead of
# -march=native so the binaries run on any current server CPU they are copied to.
# Nothing here uses the reference's autotools build.  The archive is linked whole:
# the CPU MemoryBackend registers itself from a static initialiser that a
# plain archive link would drop.

REF      ?= $(HONEI_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF=<reference checkout> or HONEI_REFERENCE)
endif
# OUT / OVERLAY: honei_b200/binding/binding.mk builds the same library into its own
# directory with a header overlay (a directory searched before the tree)
OUT      ?= oracle/_ref
OVERLAY  ?=
OBJ      := $(OUT)/obj
CXX      ?= g++
CXXFLAGS := -std=gnu++98 -O3 -march=x86-64-v3 -DHONEI_SSE -fpermissive -w -fPIC \
            $(if $(OVERLAY),-I$(OVERLAY)) -I$(REF) -DHONEI_SOURCEDIR='"$(REF)"'

UTIL_SRC := assertion barrier benchmark_info condition_variable configuration exception \
            lock log memory_arbiter memory_backend memory_pool mutex partitioner \
            profiler shared_array tags thread ticket type_traits
LA_SRC   := absolute banded_matrix banded_matrix_qx const_vector dense_matrix dense_matrix_tile \
            dense_vector dense_vector_range dense_vector_slice matrix_error sparse_matrix \
            sparse_matrix_csr sparse_matrix_ell sparse_vector vector_error \
            difference-sse dot_product-sse element_inverse-sse element_product-sse norm-sse \
            product-sse reduction-sse scale-sse scaled_sum-sse sum-sse
MC_SRC   := thread_function thread_pool ticket topology
SSE_SRC  := defect difference dot_product element_inverse element_product norm product \
            reduction scale scaled_sum sum
MATH_SRC := defect-sse

# object names carry their directory: util/ticket.cc and backends/multicore/ticket.cc collide
OBJS := $(patsubst %,$(OBJ)/util_%.o,$(UTIL_SRC)) \
        $(patsubst %,$(OBJ)/la_%.o,$(LA_SRC)) \
        $(patsubst %,$(OBJ)/mc_%.o,$(MC_SRC)) \
        $(patsubst %,$(OBJ)/sse_%.o,$(SSE_SRC)) \
        $(patsubst %,$(OBJ)/math_%.o,$(MATH_SRC))

all: $(OUT)/honei_ref

$(OBJ)/util_%.o: $(REF)/honei/util/%.cc | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/la_%.o: $(REF)/honei/la/%.cc | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/mc_%.o: $(REF)/honei/backends/multicore/%.cc | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/sse_%.o: $(REF)/honei/backends/sse/%.cc | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@
$(OBJ)/math_%.o: $(REF)/honei/math/%.cc | $(OBJ)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OBJ):
	mkdir -p $@

$(OUT)/libhonei_ref.a: $(OBJS)
	rm -f $@ && ar rcs $@ $^

$(OUT)/ref_driver.o: oracle/ref_driver.cc oracle/ref_common.hh oracle/honei_oracle.h | $(OBJ)
	$(CXX) $(CXXFLAGS) -Ioracle -c $< -o $@

# the oracle's seeded-input generator and fast ELL assembly, linked into the driver
$(OUT)/honei_oracle.o: oracle/honei_oracle.c oracle/honei_oracle.h | $(OBJ)
	gcc -std=c99 -O2 -ffp-contract=off -fPIC -c $< -o $@

$(OUT)/honei_ref: $(OUT)/ref_driver.o $(OUT)/honei_oracle.o $(OUT)/libhonei_ref.a
	$(CXX) -o $@ $(OUT)/ref_driver.o $(OUT)/honei_oracle.o -Wl,--whole-archive $(OUT)/libhonei_ref.a -Wl,--no-whole-archive -lpthread -lm

lib: $(OUT)/libhonei_ref.a

clean:
	rm -rf $(OUT)

.PHONY: all lib clean

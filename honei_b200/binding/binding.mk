# Builds the B200 tag binding against a HONEI tree and its test program:
#
#   make -f honei_b200/binding/binding.mk REF=<reference checkout> -j8   (or HONEI_REFERENCE=<checkout>)
#
# 1. a header overlay: the tree's honei/util/tags.hh with the tag value tv_b200
#    added to its TagValue enum (the one line a maintainer adds to the tree itself);
# 2. the tree's library compiled against the overlay (oracle/ref.mk, its own
#    output directory: every translation unit must see the same enum);
# 3. the binding (b200_backend.cc) and tests/cpp/binding_test.cc, warnings as
#    errors (the tree's headers are system headers here), linked with the tree,
#    libhonei_b200.so and the CUDA runtime.
# Outputs only under oracle/_ref/b200/.

REF   ?= $(HONEI_REFERENCE)
ifeq ($(strip $(REF)),)
$(error set REF=<reference checkout> or HONEI_REFERENCE)
endif
OUT   := oracle/_ref/b200
OVL   := $(OUT)/overlay
CUDA  ?= /usr/local/cuda
CXX   ?= g++
FLAGS := -std=gnu++98 -O2 -march=x86-64-v3 -DHONEI_SSE -fpermissive -fPIC -Wall -Wextra -Werror \
         -isystem $(OVL) -isystem $(REF) -isystem $(CUDA)/include -Iinclude -Ihonei_b200/binding \
         -DHONEI_SOURCEDIR='"$(REF)"'

all: $(OUT)/binding_test

$(OVL)/honei/util/tags.hh: $(REF)/honei/util/tags.hh
	mkdir -p $(dir $@)
	sed 's/^\([[:space:]]*\)tv_none$$/\1tv_b200,\n\1tv_none/' $< > $@
	grep -q 'tv_b200,' $@

$(OUT)/libhonei_ref.a: $(OVL)/honei/util/tags.hh
	$(MAKE) -f oracle/ref.mk REF=$(REF) OUT=$(OUT) OVERLAY=$(OVL) lib

$(OUT)/b200_backend.o: honei_b200/binding/b200_backend.cc honei_b200/binding/b200_operations.hh \
                       honei_b200/binding/b200_tag.hh include/honei_b200.h $(OVL)/honei/util/tags.hh
	$(CXX) $(FLAGS) -c $< -o $@

$(OUT)/binding_test.o: tests/cpp/binding_test.cc honei_b200/binding/b200_operations.hh \
                       honei_b200/binding/b200_tag.hh include/honei_b200.h $(OVL)/honei/util/tags.hh
	$(CXX) $(FLAGS) -c $< -o $@

$(OUT)/binding_test: $(OUT)/binding_test.o $(OUT)/b200_backend.o $(OUT)/libhonei_ref.a
	$(CXX) -o $@ $(OUT)/binding_test.o $(OUT)/b200_backend.o -Wl,--whole-archive $(OUT)/libhonei_ref.a \
	    -Wl,--no-whole-archive -Lhonei_b200 -lhonei_b200 -Wl,-rpath,'$$ORIGIN/../../../honei_b200' \
	    -L$(CUDA)/lib64 -lcudart -Wl,-rpath,$(CUDA)/lib64 -lpthread -lm

.PHONY: all

# Builds the B200 BFS library, its CLI and the test oracles.
#
#   beedrill_b200/lib/libbeedrill_b200.so   C ABI (include/beedrill_b200.h)
#   beedrill_b200/bin/hybrid_bfs            CLI with the reference's flags
#   beedrill_b200/bin/components            connected-components CLI, same
#   oracle/...                              see oracle/Makefile
#
# sm_100a only.  nvcc cross-compiles without a GPU.
NVCC ?= /usr/local/cuda/bin/nvcc
CXX := g++
ARCH := -gencode arch=compute_100a,code=sm_100a
NVFLAGS := -O3 -std=c++17 $(ARCH) -lineinfo -Xcompiler -fPIC -Xcompiler -Wall \
           -Iinclude -Ibeedrill_b200/csrc --expt-relaxed-constexpr
CSRC := beedrill_b200/csrc
CU_SRCS := $(CSRC)/bd_common.cu $(CSRC)/bd_graph.cu $(CSRC)/bd_bfs.cu $(CSRC)/bd_policy.cu $(CSRC)/bd_msbfs.cu \
           $(CSRC)/bd_check.cu $(CSRC)/bd_components.cu
CU_OBJS := $(patsubst $(CSRC)/%.cu,beedrill_b200/_build/%.o,$(CU_SRCS))
HDRS := include/beedrill_b200.h $(CSRC)/bd_internal.h $(CSRC)/bd_bfs_device.cuh $(CSRC)/bd_device_util.cuh \
        $(CSRC)/bd_policy.cuh
LIB := beedrill_b200/lib/libbeedrill_b200.so
CLI := beedrill_b200/bin/hybrid_bfs
CC_CLI := beedrill_b200/bin/components

all: $(LIB) $(CLI) $(CC_CLI) oracle

beedrill_b200/_build/%.o: $(CSRC)/%.cu $(HDRS)
	@mkdir -p beedrill_b200/_build
	$(NVCC) $(NVFLAGS) -c -o $@ $<

$(LIB): $(CU_OBJS)
	@mkdir -p beedrill_b200/lib
	$(NVCC) $(ARCH) -shared -o $@ $(CU_OBJS) -lcudart_static

$(CLI): $(CSRC)/hybrid_bfs_main.cc include/beedrill/hybrid_bfs.hpp $(LIB)
	@mkdir -p beedrill_b200/bin
	$(CXX) -std=c++17 -O2 -Wall -Iinclude -o $@ $(CSRC)/hybrid_bfs_main.cc \
		-Lbeedrill_b200/lib -lbeedrill_b200 -Wl,-rpath,'$$ORIGIN/../lib'

$(CC_CLI): $(CSRC)/components_main.cc include/beedrill/hybrid_bfs.hpp $(LIB)
	@mkdir -p beedrill_b200/bin
	$(CXX) -std=c++17 -O2 -Wall -Iinclude -o $@ $(CSRC)/components_main.cc \
		-Lbeedrill_b200/lib -lbeedrill_b200 -Wl,-rpath,'$$ORIGIN/../lib'

oracle:
	$(MAKE) -s -C oracle

# registers / spills / shared memory of every kernel
ptxas-report:
	@for f in $(CU_SRCS); do $(NVCC) $(NVFLAGS) -Xptxas -v -c -o /dev/null $$f 2>&1 | \
		grep -E "Compiling entry|registers|spill" ; done

clean:
	rm -rf beedrill_b200/_build $(LIB) $(CLI) $(CC_CLI)

.PHONY: all oracle clean ptxas-report

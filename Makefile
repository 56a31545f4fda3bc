# Build of the gatlas_b200 library (CUDA kernels + C ABI + C++ host), its
# command-line tools, and the oracle used by the tests.
#   make            -> gatlas_b200/lib/libgatlas_b200.so, gatlas_b200/bin/*, oracle
#   make -j8        (parallel)
NVCC    := /usr/local/cuda/bin/nvcc
CXX_SYS := g++
ARCH    := -gencode arch=compute_100a,code=sm_100a
NVFLAGS := -O3 -std=c++17 $(ARCH) -lineinfo -ccbin $(CXX_SYS) -Xcompiler -fPIC,-Wall \
           --expt-relaxed-constexpr -Iinclude
CXXFLAGS := -O2 -std=c++17 -fPIC -Wall -Wextra -Iinclude -I/usr/local/cuda/include
BUILD   := _build
LIBDIR  := gatlas_b200/lib
BINDIR  := gatlas_b200/bin
LIB     := $(LIBDIR)/libgatlas_b200.so

CU_SRC  := $(wildcard gatlas_b200/csrc/*.cu gatlas_b200/csrc/kernels/*.cu)
CPP_SRC := $(wildcard gatlas_b200/csrc/*.cpp gatlas_b200/csrc/host/*.cpp gatlas_b200/csrc/kernels/*.cpp)
CU_OBJ  := $(patsubst %.cu,$(BUILD)/%.o,$(CU_SRC))
CPP_OBJ := $(patsubst %.cpp,$(BUILD)/%.o,$(CPP_SRC))
HDRS    := $(wildcard include/*.h gatlas_b200/csrc/*.hpp gatlas_b200/csrc/*.cuh \
             gatlas_b200/csrc/kernels/*.hpp gatlas_b200/csrc/kernels/*.cuh gatlas_b200/csrc/host/*.hpp)

CLI_SRC := $(wildcard gatlas_b200/cli/*.cpp)
CLI_BIN := $(patsubst gatlas_b200/cli/%.cpp,$(BINDIR)/%,$(CLI_SRC)) $(BINDIR)/retry

all: $(LIB) $(CLI_BIN) oracle

$(BUILD)/%.o: %.cu $(HDRS)
	@mkdir -p $(dir $@)
	$(NVCC) $(NVFLAGS) -c $< -o $@

$(BUILD)/%.o: %.cpp $(HDRS)
	@mkdir -p $(dir $@)
	$(CXX_SYS) $(CXXFLAGS) -c $< -o $@

# The SIMT kernel template embedded as a string for run-time compilation.
GEN := $(BUILD)/gen
$(GEN)/gemm_simt_source.inc: gatlas_b200/csrc/kernels/gemm_simt.cuh
	@mkdir -p $(GEN)
	( printf 'R"GATLAS_SRC('; cat $<; printf ')GATLAS_SRC"\n' ) > $@

$(GEN)/gemm_image_source.inc: gatlas_b200/csrc/kernels/gemm_image.cuh
	@mkdir -p $(GEN)
	( printf 'R"GATLAS_SRC('; cat $<; printf ')GATLAS_SRC"\n' ) > $@

$(BUILD)/gatlas_b200/csrc/kernels/jit.o: gatlas_b200/csrc/kernels/jit.cpp $(GEN)/gemm_simt_source.inc \
		$(GEN)/gemm_image_source.inc $(HDRS)
	@mkdir -p $(dir $@)
	$(CXX_SYS) $(CXXFLAGS) -I$(GEN) -c $< -o $@

$(LIB): $(CU_OBJ) $(CPP_OBJ)
	@mkdir -p $(LIBDIR)
	$(NVCC) $(ARCH) -ccbin $(CXX_SYS) -shared -cudart static -o $@ $^ -lpthread -ldl -lrt

# The tools link only against the library, whose statically linked CUDA
# runtime they share (one runtime instance per process).
$(BINDIR)/%: gatlas_b200/cli/%.cpp $(LIB) $(HDRS)
	@mkdir -p $(BINDIR)
	$(CXX_SYS) $(CXXFLAGS) -Igatlas_b200/csrc -o $@ $< -L$(LIBDIR) -lgatlas_b200 -Wl,-rpath,'$$ORIGIN/../lib'

$(BINDIR)/retry: gatlas_b200/cli/retry
	@mkdir -p $(BINDIR)
	cp $< $@ && chmod +x $@

oracle:
	$(MAKE) -s -C oracle

clean:
	rm -rf $(BUILD) $(LIBDIR) $(BINDIR)
	$(MAKE) -s -C oracle clean

.PHONY: all clean oracle

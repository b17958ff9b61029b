#!/bin/sh
# Compile the reference's own CPU propagation sources (read in place under
# /root/reference, never copied) into oracle/_ref/ with the shims in
# oracle/ref_shim/: libfwi2d_ref32.so (FP32, the reference's default build)
# and libfwi2d_ref64.so (FP64, as ENABLE_DOUBLE_PRECISION).
# Flags follow the reference's CMakeLists.txt: -O3 -fopenmp, no MPI, no CUDA.
set -e
REF=${FWI2D_REFERENCE:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/_ref"
if [ ! -d "$REF/src/cpp" ]; then
    echo "reference sources not found at $REF; skipping the reference build" >&2
    exit 0
fi
mkdir -p "$OUT"
SRCS="we_op.cpp spatial_operators.cpp injector.cpp misc.cpp operator.cpp nlsolver.cpp dummy.cpp"
for prec in 32 64; do
    B="$OUT/obj$prec"
    mkdir -p "$B"
    DEF=""
    [ "$prec" = 64 ] && DEF="-DDOUBLE_PRECISION"
    OBJS=""
    for s in $SRCS; do
        o="$B/${s%.cpp}.o"
        g++ -std=c++11 -O3 -fopenmp -fPIC -fpermissive -w $DEF -I"$HERE/ref_shim" -I"$REF/src/include" -c "$REF/src/cpp/$s" -o "$o"
        OBJS="$OBJS $o"
    done
    for s in ispc_loops.cpp stubs.cpp ref_driver.cpp; do
        o="$B/${s%.cpp}.o"
        g++ -std=c++11 -O3 -fopenmp -fPIC -w $DEF -I"$HERE/ref_shim" -I"$REF/src/include" -c "$HERE/ref_shim/$s" -o "$o"
        OBJS="$OBJS $o"
    done
    g++ -shared -fopenmp -o "$OUT/libfwi2d_ref$prec.so" $OBJS -Wl,--no-undefined
done
# The reference's GPU path (src/cuda/cudaKernels.cu, cudaWeOp.cpp; the
# reference's CMake adds -DCUDA and compiles the .cu with -std=c++11 -O3 -w
# -Xcompiler -fopenmp), FP32, for sm_100a: libfwi2d_ref32_cuda.so, used only to
# time the reference's own GPU implementation beside this library.
CUDA_HOME=${CUDA_HOME:-/usr/local/cuda}
if [ -x "$CUDA_HOME/bin/nvcc" ]; then
    B="$OUT/objcuda"
    mkdir -p "$B"
    INC="-I$HERE/ref_shim -I$REF/src/include -I$REF/src/cuda -I$CUDA_HOME/include"
    OBJS=""
    for s in we_op.cpp spatial_operators.cpp injector.cpp misc.cpp operator.cpp nlsolver.cpp; do
        o="$B/${s%.cpp}.o"
        g++ -std=c++11 -O3 -fopenmp -fPIC -fpermissive -w -DCUDA $INC -c "$REF/src/cpp/$s" -o "$o"
        OBJS="$OBJS $o"
    done
    g++ -std=c++11 -O3 -fopenmp -fPIC -fpermissive -w -DCUDA $INC -c "$REF/src/cuda/cudaWeOp.cpp" -o "$B/cudaWeOp.o"
    "$CUDA_HOME/bin/nvcc" -std=c++11 -O3 -w -Xcompiler -fopenmp,-fPIC -gencode arch=compute_100a,code=sm_100a \
        $INC -c "$REF/src/cuda/cudaKernels.cu" -o "$B/cudaKernels.o"
    OBJS="$OBJS $B/cudaWeOp.o $B/cudaKernels.o"
    for s in ispc_loops.cpp stubs.cpp ref_driver.cpp; do
        o="$B/${s%.cpp}.o"
        g++ -std=c++11 -O3 -fopenmp -fPIC -w -DCUDA $INC -c "$HERE/ref_shim/$s" -o "$o"
        OBJS="$OBJS $o"
    done
    g++ -shared -fopenmp -o "$OUT/libfwi2d_ref32_cuda.so" $OBJS -L"$CUDA_HOME/lib64" -lcudart_static -ldl -lrt -lpthread \
        -Wl,--no-undefined
fi
# The reference built as its maintainer would switch it to this library:
# the same -DCUDA objects, with fwi2d_b200/integration/we_op_b200.cpp (its
# propagate_gpu hook on fwi2d_propagate) in place of src/cuda, linked with
# libfwi2d_b200.so: libfwi2d_ref32_b200.so.  The tests run the reference's own
# operator classes and solver gradient through it.
LIB="$HERE/../fwi2d_b200/libfwi2d_b200.so"
if [ -x "$CUDA_HOME/bin/nvcc" ] && [ -f "$LIB" ] && [ -d "$OUT/objcuda" ]; then
    B="$OUT/objcuda"
    INC="-I$HERE/ref_shim -I$REF/src/include -I$REF/src/cuda -I$CUDA_HOME/include -I$HERE/../include"
    g++ -std=c++11 -O3 -fopenmp -fPIC -w -DCUDA $INC -c "$HERE/../fwi2d_b200/integration/we_op_b200.cpp" \
        -o "$B/we_op_b200.o"
    OBJS=""
    for s in we_op spatial_operators injector misc operator nlsolver ispc_loops stubs ref_driver; do
        OBJS="$OBJS $B/$s.o"
    done
    g++ -shared -fopenmp -o "$OUT/libfwi2d_ref32_b200.so" $OBJS "$B/we_op_b200.o" \
        -L"$HERE/../fwi2d_b200" -lfwi2d_b200 -Wl,-rpath,'$ORIGIN/../../fwi2d_b200' -Wl,--no-undefined
fi
echo "reference oracle built in $OUT"

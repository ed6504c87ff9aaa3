# backend_nvidia.jl -- the B200 backend of LibNEGF.jl.
#
# Drop-in for src/backend_cpu.jl: LibNEGF.jl includes
# "backend_" * ENV["LIBNEGF_HW"] * ".jl" (src/LibNEGF.jl:54-56), so with
# LIBNEGF_HW=nvidia this file defines the same be_* functions, with the same
# argument orders, over device blocks.  Every computation reaches the GPU
# through ccall into libnegf_b200.so (include/negf_b200.h); CUDA.jl only
# allocates the device blocks, moves them to and from the host and supplies
# the current stream.  There is no CPU fallback: a failing call raises the
# library's error message (the reference prints and calls exit(),
# src/backend_cpu.jl:151-155).
#
# Two lines of LibNEGF.jl change with this backend: ArrayWithType
# (src/LibNEGF.jl:47) names the device matrix type, as the comment there
# anticipates for Metal, and Block.Full (src/block.jl:11) is widened from
# Array to AbstractMatrix so that selected-inverse blocks live on the device.
# The whole-sweep methods (one library call per algorithm function) are in
# backend_nvidia_sweeps.jl, included after the algorithm files.

using CUDA
using LinearAlgebra

const LIBNEGF = get(ENV, "LIBNEGF_B200_SO", joinpath(@__DIR__, "..", "libnegf_b200", "libnegf_b200.so"))
const NvMatrix = CUDA.CuMatrix{FieldType}

# The LU-like block of this backend: the library inverts the factored block
# once (blocked Gauss-Jordan with partial pivoting) and every later solve is a
# tensor-core product with that inverse.  Replaces CpuLU (backend_cpu.jl:7-10).
mutable struct NvLU
    inv::NvMatrix
end

const ArrayOrLUUnder_ = Union{NvMatrix,NvLU,Nothing}
const ArrayOrLU_ = Matrix{ArrayOrLUUnder_}
const ArrayOrLUView_ = SubArray{ArrayOrLUUnder_,2,ArrayOrLU_,Tuple{UnitRange{Int},UnitRange{Int}},false}

negf_stream() = CUDA.stream().handle

function negf_check(rc::Cint)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:negf_last_error, LIBNEGF), Cstring, ()))
    error("libnegf_b200 (code $(rc)): $(msg)")
end

# mirrors negf_zgemm_problem (include/negf_b200.h)
struct NegfGemm
    A::Ptr{Cvoid}
    B::Ptr{Cvoid}
    Cin::Ptr{Cvoid}
    C::Ptr{Cvoid}
    m::Int32
    n::Int32
    k::Int32
    lda::Int32
    ldb::Int32
    ldc::Int32
    ldcin::Int32
    alpha::NTuple{2,Float64}
    beta::NTuple{2,Float64}
    diag::NTuple{2,Float64}
end

cplx2(x::Number) = (Float64(real(x)), Float64(imag(x)))
ld(M) = Int32(max(1, stride(M, 2)))

# C = alpha op(A) op(B) + beta C + diag I, one problem
function negf_gemm!(tA::Char, tB::Char, alpha::Number, A, B, beta::Number, C::NvMatrix; diag::Number=0)
    k = A === nothing ? 0 : (tA == 'N' ? size(A, 2) : size(A, 1))
    p = Ref(NegfGemm(A === nothing ? C_NULL : pointer(A), B === nothing ? C_NULL : pointer(B),
                     beta == 0 ? C_NULL : pointer(C), pointer(C), size(C, 1), size(C, 2), k,
                     A === nothing ? 1 : ld(A), B === nothing ? 1 : ld(B), ld(C), ld(C),
                     cplx2(alpha), cplx2(beta), cplx2(diag)))
    negf_check(ccall((:negf_zgemm_batched, LIBNEGF), Cint, (Cchar, Cchar, Int32, Ptr{NegfGemm}, Ptr{Cvoid}),
                     tA, tB, 1, p, negf_stream()))
end

function negf_copy!(op::Char, Mout::NvMatrix, Min::NvMatrix)
    negf_check(ccall((:negf_zcopy_batched, LIBNEGF), Cint,
                     (Cchar, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32},
                      Ptr{Cvoid}),
                     op, 1, Int32[size(Mout, 1)], Int32[size(Mout, 2)], [pointer(Min)], Int32[ld(Min)],
                     [pointer(Mout)], Int32[ld(Mout)], negf_stream()))
end

function negf_inv!(Mout::NvMatrix, Min::NvMatrix)
    info = zeros(Int32, 1)
    negf_check(ccall((:negf_zinv_batched, LIBNEGF), Cint,
                     (Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Int32},
                      Ptr{Cvoid}),
                     1, Int32[size(Min, 1)], [pointer(Min)], Int32[ld(Min)], [pointer(Mout)], Int32[ld(Mout)], info,
                     negf_stream()))
    return info[1]
end

# ----------------------------------------------------
# 'base' types (backend_cpu.jl:26-89)

be_copy_to_hw!(Mout::NvMatrix, Min::Array) = copyto!(Mout, Min)
be_copy_to_hw(M::Array)::NvMatrix = NvMatrix(M)
be_copy_from_hw!(Mout::Array, Min::NvMatrix) = copyto!(Mout, Min)
be_copy_from_hw(M::NvMatrix)::Array = Array(M)
be_copy_in_hw!(Mout::NvMatrix, Min::NvMatrix) = negf_copy!('N', Mout, Min)

function be_copy_in_hw(M::NvMatrix)::NvMatrix
    Mout = NvMatrix(undef, size(M))
    negf_copy!('N', Mout, M)
    return Mout
end

function be_zero_array(dimsOfArr::Tuple{Int,Int})::NvMatrix
    M = NvMatrix(undef, dimsOfArr)
    negf_gemm!('N', 'N', 0, nothing, nothing, 0, M)  # k = 0: C = 0
    return M
end

function be_identity(n::Int)::NvMatrix
    M = NvMatrix(undef, (n, n))
    negf_gemm!('N', 'N', 0, nothing, nothing, 0, M; diag=1)  # k = 0: C = I
    return M
end

be_ctranspose!(Mout::NvMatrix, Min::NvMatrix, td::TimingData, cd::CountingData) = negf_copy!('C', Mout, Min)

function be_ctranspose(Min::NvMatrix, td::TimingData, cd::CountingData)::NvMatrix
    Mout = NvMatrix(undef, (size(Min, 2), size(Min, 1)))
    negf_copy!('C', Mout, Min)
    return Mout
end

# synthetic data is drawn on the host, as the reference's rand, then copied
be_random_array(dimsOfArr::Tuple{Int,Int})::NvMatrix = NvMatrix(rand(FieldType, dimsOfArr))

function be_fill!(M::NvMatrix, x::Number)
    negf_check(ccall((:negf_zfill_batched, LIBNEGF), Cint,
                     (Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Float64}, Ptr{Cvoid}),
                     1, Int32[size(M, 1)], Int32[size(M, 2)], [pointer(M)], Int32[ld(M)], collect(cplx2(x)),
                     negf_stream()))
end

# ----------------------------------------------------
# composite types (backend_cpu.jl:95-141)

# A = inverse of the stored inverse (not for performance, as in the reference)
function be_A_from_LU(M::NvLU)::NvMatrix
    A = NvMatrix(undef, size(M.inv))
    negf_check(negf_inv!(A, M.inv) == 0 ? Cint(0) : Cint(3))
    return A
end

be_zero_lu(n::Int)::NvLU = NvLU(be_zero_array((n, n)))

# ----------------------------------------------------
# functionality (backend_cpu.jl:143-289)

function be_inv(M::NvMatrix)::NvMatrix
    Mout = NvMatrix(undef, size(M))
    negf_check(negf_inv!(Mout, M) == 0 ? Cint(0) : Cint(3))
    return Mout
end

function be_lu!(Mout::NvLU, Min::NvMatrix, td::TimingData, cd::CountingData)
    negf_inv!(Mout.inv, Min) == 0 || error("libnegf_b200: zero pivot in the LU of a diagonal block")
end

function be_lu(M::NvMatrix, td::TimingData, cd::CountingData)::NvLU
    Mlu = be_zero_lu(size(M, 1))
    be_lu!(Mlu, M, td, cd)
    return Mlu
end

be_inv_from_lu!(Mout::NvMatrix, Min::NvLU) = negf_copy!('N', Mout, Min.inv)

# getrs with a precomputed LU: Mout = op(X)^{-1} Min = op(X^{-1}) Min
be_mldivide!(trans::Char, Mout::NvMatrix, Min::NvMatrix, Mlu::NvLU, td::TimingData, cd::CountingData) =
    negf_gemm!(trans == 'N' ? 'N' : 'C', 'N', 1, Mlu.inv, Min, 0, Mout)

be_gemm!(tA::Char, tB::Char, alpha::Number, A::NvMatrix, B::NvMatrix, beta::Number, C::NvMatrix,
         td::TimingData, cd::CountingData) = negf_gemm!(tA, tB, alpha, A, B, beta, C)

function be_mul(M1::NvMatrix, M2::NvMatrix)::NvMatrix
    C = NvMatrix(undef, (size(M1, 1), size(M2, 2)))
    negf_gemm!('N', 'N', 1, M1, M2, 0, C)
    return C
end

# getri with identity pivots: A (L\U factors) <- U^{-1} L^{-1}
be_getri!(A::NvMatrix, td::TimingData, cd::CountingData) =
    negf_check(ccall((:negf_zgetri_nopiv_batched, LIBNEGF), Cint,
                     (Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Cvoid}),
                     1, Int32[size(A, 1)], [pointer(A)], Int32[ld(A)], negf_stream()))

function be_trsm!(side::Char, ul::Char, tA::Char, dA::Char, alpha::Number, A::NvMatrix, B::NvMatrix,
                  td::TimingData, cd::CountingData)
    negf_check(ccall((:negf_ztrsm_batched, LIBNEGF), Cint,
                     (Cchar, Cchar, Cchar, Cchar, Ptr{Float64}, Int32, Ptr{Int32}, Ptr{Int32}, Ptr{Ptr{Cvoid}},
                      Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Cvoid}),
                     side, ul, tA, dA, collect(cplx2(alpha)), 1, Int32[size(B, 1)], Int32[size(B, 2)],
                     [pointer(A)], Int32[ld(A)], [pointer(B)], Int32[ld(B)], negf_stream()))
end

# getrf whose pivots are discarded, as LinearAlgebra.LAPACK.getrf!(A, ipiv) is
# used by the reference (backend_cpu.jl:255-265)
function be_getrf!(A::NvMatrix, td::TimingData, cd::CountingData)
    info = zeros(Int32, 1)
    negf_check(ccall((:negf_zgetrf_batched, LIBNEGF), Cint,
                     (Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Int32}, Ptr{Cvoid}),
                     1, Int32[size(A, 1)], [pointer(A)], Int32[ld(A)], [C_NULL], info, negf_stream()))
end

# be_potrf! and be_herk! (backend_cpu.jl:267-289) are not called by any
# LibNEGF.jl algorithm; the library provides no Cholesky factorisation.
be_potrf!(uplo::Char, A::NvMatrix, td::TimingData, cd::CountingData) =
    error("libnegf_b200 provides no Cholesky factorisation (be_potrf! is unused by the LibNEGF.jl algorithms)")

# C = alpha op(A) op(A)^H + beta C over the whole matrix (the triangle uplo is
# the Hermitian result; the other triangle is written too)
be_herk!(uplo::Char, tA::Char, alpha::Number, A::NvMatrix, beta::Number, C::NvMatrix, td::TimingData,
         cd::CountingData) = negf_gemm!(tA, tA == 'N' ? 'C' : 'N', alpha, A, A, beta, C)

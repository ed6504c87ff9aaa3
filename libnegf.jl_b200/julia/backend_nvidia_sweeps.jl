# backend_nvidia_sweeps.jl -- whole-sweep methods of the B200 backend.
#
# Included after the algorithm files (after src/selected_inverse.jl in
# src/LibNEGF.jl) when LIBNEGF_HW=nvidia, so that these definitions replace
# the generic ones: each reference algorithm function becomes ONE library
# call that runs the whole sweep as batched launches on the device, instead of
# a sequence of per-block be_* calls.  Same signatures, inputs and outputs as
# the functions they replace (cited at each method).  Needs backend_nvidia.jl.

# device pointers of a BlockMatrix's tridiagonal (1-based layers)
_diag_ptrs(M::BlockMatrix) = Ptr{Cvoid}[pointer(M.M[i, i]) for i in 1:length(M.blockSizes)]
_up_ptrs(M::BlockMatrix) = Ptr{Cvoid}[pointer(M.M[i, i+1]) for i in 1:length(M.blockSizes)-1]
_lo_ptrs(M::BlockMatrix) = Ptr{Cvoid}[pointer(M.M[i+1, i]) for i in 1:length(M.blockSizes)-1]

# src/matinvertndiag_rgf.jl:114-200 (with buildFullInv, every block of Mout)
function bndiag_of_inv_rgf_local!(Mout::BlockMatrix, Min::BlockMatrix, auxData::AuxDataRGF, td::TimingData,
                                  cd::CountingData)
    npl = length(Min.blockSizes)
    full = C_NULL
    if auxData.buildFullInv
        full = Ptr{Cvoid}[isassigned(Mout.M, i, j) && Mout.M[i, j] !== nothing ? pointer(Mout.M[i, j]) : C_NULL
                          for j in 1:npl for i in 1:npl]
        full = permutedims(reshape(full, npl, npl))[:]  # row-major block index i*npl + j
    end
    negf_check(ccall((:negf_rgf, LIBNEGF), Cint,
                     (Int32, Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}},
                      Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
                     1, npl, Int32.(Min.blockSizes), _diag_ptrs(Min), _up_ptrs(Min), _lo_ptrs(Min),
                     _diag_ptrs(Mout), _up_ptrs(Mout), _lo_ptrs(Mout), full, negf_stream()))
end

# src/matinvertndiag_ddrgf_core.jl:32-46 (the same sweep)
bndiag_of_inv_rgf_global!(Mout::BlockMatrix, Min::BlockMatrix, auxData::AuxDataRGF, td::TimingData,
                          cd::CountingData) = bndiag_of_inv_rgf_local!(Mout, Min, auxData, td, cd)

# src/keldyshndiag.jl:120-164: G^n = M^{-1} S M^{-H} into auxData.buffS
function keldyshndiag!(M::BlockMatrix, S::BlockMatrix, auxData::AuxDataKeldysh, td::TimingData, cd::CountingData)
    npl = length(M.blockSizes)
    bm_copy!(auxData.buffS, S)
    negf_check(ccall((:negf_keldysh, LIBNEGF), Cint,
                     (Int32, Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}},
                      Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
                     1, npl, Int32.(M.blockSizes), _diag_ptrs(M), _up_ptrs(M), _lo_ptrs(M),
                     _diag_ptrs(auxData.buffS), _up_ptrs(auxData.buffS), negf_stream()))
end

# src/matinvertndiag_general_rgf.jl:31-146: the band of M^{-1} into Mout
function bndiag_of_inv_general_rgf!(Mout::BlockMatrix, Min::BlockMatrix, auxData::AuxDataRGF, td::TimingData,
                                    cd::CountingData)
    npl = length(Min.blockSizes)
    ndiag = Min.ndiag["in"]
    w = (ndiag - 1) ÷ 2
    band(M) = Ptr{Cvoid}[abs(i - j) <= w ? pointer(M.M[i, j]) : C_NULL for i in 1:npl for j in 1:npl]
    negf_check(ccall((:negf_general_rgf, LIBNEGF), Cint,
                     (Int32, Int32, Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
                     1, npl, ndiag, Int32.(Min.blockSizes), band(Min), band(Mout), negf_stream()))
end

# src/selected_inverse.jl:9-55 and :139-206 on a Matrix{Block} (uniform block
# size; fill-in blocks are created zeroed before the call, as :41-46 does)
function _selinv!(A::Matrix, mode::Int32)
    npl = size(A, 1)
    b = A[1, 1].row
    if mode & 1 != 0
        for i in 1:npl, k in i+1:npl, l in k+1:npl
            if isassigned(A, i, k) && isassigned(A, i, l) && !isassigned(A, k, l)
                A[k, l] = Block(be_zero_array((b, b)))
                A[l, k] = Block(be_zero_array((b, b)))
            end
        end
    end
    tab = Ptr{Cvoid}[isassigned(A, i, j) ? pointer(A[i, j].Full) : C_NULL for i in 1:npl for j in 1:npl]
    fill = zeros(UInt8, npl * npl)
    negf_check(ccall((:negf_selected_inverse, LIBNEGF), Cint,
                     (Int32, Int32, Ptr{Ptr{Cvoid}}, Ptr{UInt8}, Int32, Ptr{Cvoid}),
                     npl, b, tab, fill, mode, negf_stream()))
    return A
end
Block_factorization!(A::Matrix, td::TimingData, cd::CountingData) = _selinv!(A, Int32(1))
Block_inverse!(A::Matrix, td::TimingData, cd::CountingData) = _selinv!(A, Int32(2))

# src/matinvertndiag_ddrgf_core.jl:719-758 over all levels of listOfAuxData
# (the Schur complement recursion of :656-680 runs inside the library)
function bndiag_of_inv_ddrgf!(Min::BlockMatrix, listOfAuxData::Vector{AuxDataDDRGF}, td::TimingData,
                              cd::CountingData, depth::Int)
    npl = length(Min.blockSizes)
    out = listOfAuxData[depth].buffMout
    d1 = Int32[a.blockSizeD1 for a in listOfAuxData[depth:end] if a.nrTasks > 1]
    negf_check(ccall((:negf_ddrgf_levels, LIBNEGF), Cint,
                     (Int32, Int32, Ptr{Int32}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Int32, Ptr{Int32},
                      Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Ptr{Cvoid}}, Ptr{Cvoid}),
                     1, npl, Int32.(Min.blockSizes), _diag_ptrs(Min), _up_ptrs(Min), _lo_ptrs(Min),
                     length(d1), isempty(d1) ? C_NULL : d1,
                     _diag_ptrs(out), _up_ptrs(out), _lo_ptrs(out), negf_stream()))
end

# src/matinvertndiag_ddrgf_utils.jl:357-453: the partition search, in the library
function opt_params(Min::BlockMatrix, rLU::Float64, rMLDIV::Float64, dampRGF::Float64)
    nl = Ref{Int32}(0)
    tasks = zeros(Int32, 6)
    d1 = zeros(Int32, 6)
    cost = Ref{Float64}(0)
    negf_check(ccall((:negf_ddrgf_opt_params, LIBNEGF), Cint,
                     (Int32, Int32, Float64, Float64, Float64, Ref{Int32}, Ptr{Int32}, Ptr{Int32}, Ref{Float64}),
                     length(Min.blockSizes), Threads.nthreads(), rLU, rMLDIV, dampRGF, nl, tasks, d1, cost))
    return Int(nl[]), Int.(tasks[1:nl[]]), Int.(d1[1:nl[]]), cost[]
end

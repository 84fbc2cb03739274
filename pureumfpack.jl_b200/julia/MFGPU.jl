# MFGPU.jl -- ccall shim that routes PureUMFPACK.jl's multifrontal path to
# libmfgpu.so (include/mfgpu.h).  Drop this file into the reference package
# (e.g. src/mfgpu.jl, `include("mfgpu.jl")` after "multifrontal.jl") and set
# ENV["PUREUMFPACK_MFGPU"] to the library path.  The host keeps the
# reference's own ordering, scaling and symbolic analysis (symbolic_mf); the
# numeric factorization and the solves run on the GPU.
#
# Not executed in the build image (no Julia toolchain there); the Python
# binding pureumfpack/_lib.py drives the same symbols and is what the tests run.

module MFGPU

using SparseArrays: SparseMatrixCSC, nonzeros, rowvals
using LinearAlgebra: SingularException
using Libdl

const libmfgpu = get(ENV, "PUREUMFPACK_MFGPU", joinpath(@__DIR__, "..", "pureumfpack", "libmfgpu.so"))

mutable struct Handle
    ptr::Ptr{Cvoid}
    n::Int
    f32::Bool   # the last factorization is of a Float32 matrix
    c64::Bool   # the last factorization is of a ComplexF64 matrix
end

# The C ABI takes Int64 indices; a SparseMatrixCSC{Tv, Int32} (the reference's
# generic Ti, test/robustness.jl) is widened on the way in and its factors
# are returned with the caller's index type.
_i64(v::Vector{Int64}) = v
_i64(v::AbstractVector{<:Integer}) = Vector{Int64}(v)
_ti(::Type{Int64}, v::Vector{Int64}) = v
_ti(::Type{Ti}, v::Vector{Int64}) where {Ti <: Integer} = Vector{Ti}(v)

function _check(h::Handle, rc::Cint)
    rc >= 0 && return Int(rc)
    msg = unsafe_string(ccall((:mfgpu_last_error, libmfgpu), Cstring, (Ptr{Cvoid},), h.ptr))
    rc == -1 && throw(ArgumentError(msg))
    rc == -6 && throw(DimensionMismatch(msg))
    error("libmfgpu error $rc: $msg")
end

function create(; device::Integer = 0, precision::Integer = 0)
    opts = Ref((Int32(device), Int32(precision), Int32(0), Int32(0)))
    out = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:mfgpu_create, libmfgpu), Cint, (Ref{NTuple{4, Int32}}, Ref{Ptr{Cvoid}}), opts, out)
    rc == 0 || error("mfgpu_create failed ($rc)")
    h = Handle(out[], 0, false, false)
    finalizer(x -> ccall((:mfgpu_destroy, libmfgpu), Cvoid, (Ptr{Cvoid},), x.ptr), h)
    return h
end

# mfgpu_analyze from the reference's SymbolicMF (src/symbolic.jl:203-209):
# update set of supernode s = colstruct[sstart[s+1]-1].
function analyze!(h::Handle, A::SparseMatrixCSC{<:Union{Float64, Float32, ComplexF64}, <:Integer}, S)
    n = size(A, 2)
    nsuper = length(S.sstart) - 1
    upd_ptr = Vector{Int64}(undef, nsuper + 1)
    upd_ptr[1] = 1
    for s in 1:nsuper
        upd_ptr[s + 1] = upd_ptr[s] + length(S.colstruct[S.sstart[s + 1] - 1])
    end
    upd_idx = Vector{Int64}(undef, upd_ptr[end] - 1)
    for s in 1:nsuper
        copyto!(upd_idx, upd_ptr[s], S.colstruct[S.sstart[s + 1] - 1], 1, upd_ptr[s + 1] - upd_ptr[s])
    end
    rc = ccall((:mfgpu_analyze, libmfgpu), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{Int64}),
        h.ptr, n, _i64(A.colptr), _i64(rowvals(A)), collect(Int64, S.qf), collect(Int64, S.parent), nsuper,
        collect(Int64, S.sstart), upd_ptr, upd_idx)
    _check(h, rc)
    h.n = n
    return h
end

# Numeric factorization of Diagonal(Rs) * A (Rs === nothing: no scaling).
function factor!(h::Handle, A::SparseMatrixCSC{Float64, <:Integer}, Rs, check::Bool)
    rs = Rs === nothing ? C_NULL : pointer(Rs)
    rc = GC.@preserve Rs ccall((:mfgpu_factor, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32),
        h.ptr, nonzeros(A), rs, Int32(check))
    st = _check(h, rc)
    st > 0 && throw(Main.LinearAlgebra.SingularException(st))
    h.f32 = false
    h.c64 = false
    return h
end

# Float32 matrices (the reference's generic Tv = Float32): Float32 values,
# Rs, factors, right-hand sides and solutions.
function factor!(h::Handle, A::SparseMatrixCSC{Float32, <:Integer}, Rs, check::Bool)
    rs = Rs === nothing ? C_NULL : pointer(Rs)
    rc = GC.@preserve Rs ccall((:mfgpu_factor_f32, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{Float32}, Ptr{Float32}, Int32),
        h.ptr, nonzeros(A), rs, Int32(check))
    st = _check(h, rc)
    st > 0 && throw(Main.LinearAlgebra.SingularException(st))
    h.f32 = true
    h.c64 = false
    return h
end

# ComplexF64 matrices (the reference's generic Tv = ComplexF64): complex
# values, factors, right-hand sides and solutions in Julia's own layout; real
# Rs (row_scaling with R = real(Tv)).
function factor!(h::Handle, A::SparseMatrixCSC{ComplexF64, <:Integer}, Rs, check::Bool)
    rs = Rs === nothing ? C_NULL : pointer(Rs)
    rc = GC.@preserve Rs ccall((:mfgpu_factor_c64, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{ComplexF64}, Ptr{Float64}, Int32),
        h.ptr, nonzeros(A), rs, Int32(check))
    st = _check(h, rc)
    st > 0 && throw(Main.LinearAlgebra.SingularException(st))
    h.f32 = false
    h.c64 = true
    return h
end

# GPLUFactorization fields (src/gplu.jl:45-51) copied back from the GPU, with
# index type Ti (that of the factored matrix).
function factors(h::Handle; indextype::Type{<:Integer} = Int64)
    h.f32 && return factors_f32(h; indextype = indextype)
    h.c64 && return factors_c64(h; indextype = indextype)
    sz = Vector{Int64}(undef, 3)
    _check(h, ccall((:mfgpu_factor_sizes, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{Int64}), h.ptr, sz))
    n, nl, nu = sz
    Lp = Vector{Int64}(undef, n + 1); Li = Vector{Int64}(undef, nl); Lx = Vector{Float64}(undef, nl)
    Up = Vector{Int64}(undef, n + 1); Ui = Vector{Int64}(undef, nu); Ux = Vector{Float64}(undef, nu)
    p = Vector{Int64}(undef, n); q = Vector{Int64}(undef, n); pinv = Vector{Int64}(undef, n)
    _check(h, ccall((:mfgpu_get_factors, libmfgpu), Cint,
        (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}, Ptr{Int64}, Ptr{Int64}, Ptr{Float64}, Ptr{Int64},
         Ptr{Int64}, Ptr{Int64}), h.ptr, Lp, Li, Lx, Up, Ui, Ux, p, q, pinv))
    T = indextype
    return SparseMatrixCSC(n, n, _ti(T, Lp), _ti(T, Li), Lx), SparseMatrixCSC(n, n, _ti(T, Up), _ti(T, Ui), Ux),
           _ti(T, p), _ti(T, q), _ti(T, pinv)
end

function factors_f32(h::Handle; indextype::Type{<:Integer} = Int64)
    sz = Vector{Int64}(undef, 3)
    _check(h, ccall((:mfgpu_factor_sizes, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{Int64}), h.ptr, sz))
    n, nl, nu = sz
    Lp = Vector{Int64}(undef, n + 1); Li = Vector{Int64}(undef, nl); Lx = Vector{Float32}(undef, nl)
    Up = Vector{Int64}(undef, n + 1); Ui = Vector{Int64}(undef, nu); Ux = Vector{Float32}(undef, nu)
    p = Vector{Int64}(undef, n); q = Vector{Int64}(undef, n); pinv = Vector{Int64}(undef, n)
    _check(h, ccall((:mfgpu_get_factors_f32, libmfgpu), Cint,
        (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int64}, Ptr{Float32}, Ptr{Int64}, Ptr{Int64}, Ptr{Float32}, Ptr{Int64},
         Ptr{Int64}, Ptr{Int64}), h.ptr, Lp, Li, Lx, Up, Ui, Ux, p, q, pinv))
    T = indextype
    return SparseMatrixCSC(n, n, _ti(T, Lp), _ti(T, Li), Lx), SparseMatrixCSC(n, n, _ti(T, Up), _ti(T, Ui), Ux),
           _ti(T, p), _ti(T, q), _ti(T, pinv)
end

function factors_c64(h::Handle; indextype::Type{<:Integer} = Int64)
    sz = Vector{Int64}(undef, 3)
    _check(h, ccall((:mfgpu_factor_sizes, libmfgpu), Cint, (Ptr{Cvoid}, Ptr{Int64}), h.ptr, sz))
    n, nl, nu = sz
    Lp = Vector{Int64}(undef, n + 1); Li = Vector{Int64}(undef, nl); Lx = Vector{ComplexF64}(undef, nl)
    Up = Vector{Int64}(undef, n + 1); Ui = Vector{Int64}(undef, nu); Ux = Vector{ComplexF64}(undef, nu)
    p = Vector{Int64}(undef, n); q = Vector{Int64}(undef, n); pinv = Vector{Int64}(undef, n)
    _check(h, ccall((:mfgpu_get_factors_c64, libmfgpu), Cint,
        (Ptr{Cvoid}, Ptr{Int64}, Ptr{Int64}, Ptr{ComplexF64}, Ptr{Int64}, Ptr{Int64}, Ptr{ComplexF64}, Ptr{Int64},
         Ptr{Int64}, Ptr{Int64}), h.ptr, Lp, Li, Lx, Up, Ui, Ux, p, q, pinv))
    T = indextype
    return SparseMatrixCSC(n, n, _ti(T, Lp), _ti(T, Li), Lx), SparseMatrixCSC(n, n, _ti(T, Up), _ti(T, Ui), Ux),
           _ti(T, p), _ti(T, q), _ti(T, pinv)
end

function solve(h::Handle, B::AbstractVecOrMat{ComplexF64}; refine::Integer = 0)
    Bc = Matrix{ComplexF64}(reshape(B, size(B, 1), :))
    X = similar(Bc)
    _check(h, ccall((:mfgpu_solve_c64, libmfgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{ComplexF64}, Ptr{ComplexF64}, Int32),
        h.ptr, size(Bc, 2), Bc, X, Int32(refine)))
    return B isa AbstractVector ? vec(X) : X
end

function solve(h::Handle, B::AbstractVecOrMat{Float32}; refine::Integer = 0)
    Bc = Matrix{Float32}(reshape(B, size(B, 1), :))
    X = similar(Bc)
    _check(h, ccall((:mfgpu_solve_f32, libmfgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{Float32}, Ptr{Float32}, Int32),
        h.ptr, size(Bc, 2), Bc, X, Int32(refine)))
    return B isa AbstractVector ? vec(X) : X
end

# solve(F, b; refine) for a vector or an n x k matrix of right-hand sides.
function solve(h::Handle, B::AbstractVecOrMat{Float64}; refine::Integer = 0)
    Bc = Matrix{Float64}(reshape(B, size(B, 1), :))
    X = similar(Bc)
    n = size(Bc, 1)
    _check(h, ccall((:mfgpu_solve, libmfgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Int32),
        h.ptr, size(Bc, 2), Bc, n, X, n, Int32(refine)))
    return B isa AbstractVector ? vec(X) : X
end

# factor!(h, A, Rs, check) followed by solve(h, B; refine) in one call: the
# right-hand sides cross the bus while the GPU factors.  Returns X.
function factor_solve!(h::Handle, A::SparseMatrixCSC{Float64, <:Integer}, Rs, B::AbstractVecOrMat{Float64};
                       refine::Integer = 0, check::Bool = true)
    rs = Rs === nothing ? C_NULL : pointer(Rs)
    Bc = Matrix{Float64}(reshape(B, size(B, 1), :))
    X = similar(Bc)
    n = size(Bc, 1)
    rc = GC.@preserve Rs ccall((:mfgpu_factor_solve, libmfgpu), Cint,
        (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32, Int64, Ptr{Float64}, Int64, Ptr{Float64}, Int64, Int32),
        h.ptr, nonzeros(A), rs, Int32(check), size(Bc, 2), Bc, n, X, n, Int32(refine))
    st = _check(h, rc)
    st > 0 && throw(Main.LinearAlgebra.SingularException(st))
    h.f32 = false
    h.c64 = false
    return B isa AbstractVector ? vec(X) : X
end

# --- batched systems (many independent systems through one handle) -------
# ordering: 0 = AMD (as splu(A; method=:multifrontal)), 1 = COLAMD.
function batch_analyze!(h::Handle, As::AbstractVector{<:SparseMatrixCSC{Float64, <:Integer}}; ordering::Integer = 0)
    ns = Int64[size(A, 1) for A in As]
    cols = [_i64(A.colptr) for A in As]
    rows = [_i64(rowvals(A)) for A in As]
    cps = Ptr{Int64}[pointer(c) for c in cols]
    rvs = Ptr{Int64}[pointer(r) for r in rows]
    GC.@preserve cols rows _check(h, ccall((:mfgpu_batch_analyze, libmfgpu), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Ptr{Int64}}, Ptr{Ptr{Int64}}, Int32),
        h.ptr, length(As), ns, cps, rvs, Int32(ordering)))
    return h
end

# Factor every system with its own row scaling (scale: 0 none, 1 sum, 2 max);
# returns each system's first singular column (0 = nonsingular).
function batch_factor!(h::Handle, As::AbstractVector{<:SparseMatrixCSC{Float64, <:Integer}}; scale::Integer = 1)
    vals = Ptr{Float64}[pointer(nonzeros(A)) for A in As]
    status = zeros(Int64, length(As))
    GC.@preserve As _check(h, ccall((:mfgpu_batch_factor, libmfgpu), Cint,
        (Ptr{Cvoid}, Ptr{Ptr{Float64}}, Int32, Int32, Ptr{Int64}), h.ptr, vals, Int32(scale), Int32(0), status))
    return status
end

function batch_solve(h::Handle, Bs::Vector{Matrix{Float64}}; refine::Integer = 0)
    Xs = [similar(B) for B in Bs]
    GC.@preserve Bs Xs _check(h, ccall((:mfgpu_batch_solve, libmfgpu), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Ptr{Float64}}, Ptr{Ptr{Float64}}, Int32),
        h.ptr, size(Bs[1], 2), Ptr{Float64}[pointer(B) for B in Bs], Ptr{Float64}[pointer(X) for X in Xs],
        Int32(refine)))
    return Xs
end

# --- Gilbert-Peierls LU (gplu, splu(A; method=:gplu)) on the GPU -----------
# A separate handle type; one warp factors one system, factors and solutions
# are bit for bit the reference's gplu / solve.  The reference's splu keeps
# its own ordering (amd_order_sym / colamd_order) and row scaling and hands
# q and Rs over, e.g. in src/interface.jl's :gplu branch:
#     g = MFGPU.gplu_create(); MFGPU.gplu_factor!(g, [A], [q]; rs = [Rs], tol = tol, check = check)
#     L, U, p, q, pinv = MFGPU.gplu_factors(g, 1; indextype = Ti)
mutable struct GpluHandle
    ptr::Ptr{Cvoid}
    ns::Vector{Int}
    T::DataType    # element type of the last factorization
end

function _gcheck(g::GpluHandle, rc::Cint)
    rc >= 0 && return Int(rc)
    msg = unsafe_string(ccall((:mfgpu_gplu_last_error, libmfgpu), Cstring, (Ptr{Cvoid},), g.ptr))
    rc == -1 && throw(ArgumentError(msg))
    rc == -6 && throw(DimensionMismatch(msg))
    error("libmfgpu error $rc: $msg")
end

function gplu_create(; device::Integer = 0)
    ptr = Ref{Ptr{Cvoid}}(C_NULL)
    rc = ccall((:mfgpu_gplu_create, libmfgpu), Cint, (Int32, Ref{Ptr{Cvoid}}), Int32(device), ptr)
    rc == 0 || error("mfgpu_gplu_create failed ($rc): needs a B200 / sm_100 device")
    g = GpluHandle(ptr[], Int[], Float64)
    finalizer(x -> ccall((:mfgpu_gplu_destroy, libmfgpu), Cvoid, (Ptr{Cvoid},), x.ptr), g)
    return g
end

# The C entry points of each element type (the reference's generic Tv):
# values, Rs (real(Tv)) and the suffix of the factor / get / solve symbols.
_gsuffix(::Type{Float64}) = ""
_gsuffix(::Type{Float32}) = "_f32"
_gsuffix(::Type{ComplexF64}) = "_c64"
_gsym(base::String, T::DataType) = Symbol(base * _gsuffix(T))

# gplu(rs[i] .* As[i]; q = qs[i], tol, check, sort_factors) for every
# system, all of one element type Tv (Float64, Float32 or ComplexF64);
# throws SingularException(k) for the first singular system under check.
function gplu_factor!(g::GpluHandle, As::AbstractVector{<:SparseMatrixCSC{Tv, <:Integer}},
                      qs::AbstractVector; rs = nothing, tol::Real = 0.1, check::Bool = true,
                      sort_factors::Bool = true) where {Tv <: Union{Float64, Float32, ComplexF64}}
    ns = Int64[size(A, 1) for A in As]
    cols = [_i64(A.colptr) for A in As]
    rows = [_i64(rowvals(A)) for A in As]
    qv = [_i64(q) for q in qs]
    status = zeros(Int64, length(As))
    R = real(Tv)
    rsp = rs === nothing ? Ptr{R}[C_NULL for _ in As] : Ptr{R}[pointer(r) for r in rs]
    fn = _gsym("mfgpu_gplu_factor", Tv)
    GC.@preserve As cols rows qv rs _gcheck(g, ccall(Libdl.dlsym(_libhandle(), fn), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Ptr{Int64}}, Ptr{Ptr{Int64}}, Ptr{Ptr{Tv}}, Ptr{Ptr{Int64}},
         Ptr{Ptr{R}}, Float64, Int32, Int32, Ptr{Int64}),
        g.ptr, length(As), ns, Ptr{Int64}[pointer(c) for c in cols], Ptr{Int64}[pointer(r) for r in rows],
        Ptr{Tv}[pointer(nonzeros(A)) for A in As], Ptr{Int64}[pointer(q) for q in qv], rsp,
        Float64(tol), Int32(check), Int32(sort_factors), status))
    g.ns = Int.(ns)
    g.T = Tv
    k = findfirst(>(0), status)
    k === nothing || throw(SingularException(Int(status[k])))
    return g
end

# GPLUFactorization fields (src/gplu.jl:45-51) of system i (1-based), with
# index type Ti (that of the factored matrix: an Int32 matrix gets Int32
# factors and permutations, test/robustness.jl:27-36).
function gplu_factors(g::GpluHandle, i::Integer = 1; indextype::Type{<:Integer} = Int64)
    T = g.T
    sz = Vector{Int64}(undef, 3)
    _gcheck(g, ccall((:mfgpu_gplu_sizes, libmfgpu), Cint, (Ptr{Cvoid}, Int64, Ptr{Int64}), g.ptr, i - 1, sz))
    n, nl, nu = sz
    Lp = Vector{Int64}(undef, n + 1); Li = Vector{Int64}(undef, nl); Lx = Vector{T}(undef, nl)
    Up = Vector{Int64}(undef, n + 1); Ui = Vector{Int64}(undef, nu); Ux = Vector{T}(undef, nu)
    p = Vector{Int64}(undef, n); q = Vector{Int64}(undef, n); pinv = Vector{Int64}(undef, n)
    _gcheck(g, ccall(Libdl.dlsym(_libhandle(), _gsym("mfgpu_gplu_get_factors", T)), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Int64}, Ptr{Int64}, Ptr{T}, Ptr{Int64}, Ptr{Int64}, Ptr{T}, Ptr{Int64},
         Ptr{Int64}, Ptr{Int64}), g.ptr, i - 1, Lp, Li, Lx, Up, Ui, Ux, p, q, pinv))
    Ti = indextype
    return SparseMatrixCSC(n, n, _ti(Ti, Lp), _ti(Ti, Li), Lx), SparseMatrixCSC(n, n, _ti(Ti, Up), _ti(Ti, Ui), Ux),
           _ti(Ti, p), _ti(Ti, q), _ti(Ti, pinv)
end

# solve(F_i, b_i; refine) for every system (PureLU semantics when the
# systems were factored with rs, the raw F \ b otherwise), in the factors'
# element type.
function gplu_solve(g::GpluHandle, Bs::Vector{<:Matrix}; refine::Integer = 0)
    T = g.T
    Bt = [Matrix{T}(B) for B in Bs]
    Xs = [similar(B) for B in Bt]
    GC.@preserve Bt Xs _gcheck(g, ccall(Libdl.dlsym(_libhandle(), _gsym("mfgpu_gplu_solve", T)), Cint,
        (Ptr{Cvoid}, Int64, Ptr{Ptr{T}}, Ptr{Ptr{T}}, Int32),
        g.ptr, size(Bt[1], 2), Ptr{T}[pointer(B) for B in Bt], Ptr{T}[pointer(X) for X in Xs], Int32(refine)))
    return Xs
end

const _LIBHANDLE = Ref{Ptr{Cvoid}}(C_NULL)
function _libhandle()
    _LIBHANDLE[] == C_NULL && (_LIBHANDLE[] = Libdl.dlopen(libmfgpu))
    return _LIBHANDLE[]
end

end # module

# --- the reference-side change (in src/interface.jl / src/multifrontal.jl) ---
#
#   struct GPUPureLU{Tv,Ti,Tr}  # PureLU plus the device handle
#       F::PureLU{Tv,Ti,Tr}
#       h::MFGPU.Handle
#   end
#
#   # splu(A; method=:multifrontal) branch (src/interface.jl:103-105):
#   S = symbolic_mf(A)                       # the reference's own host code
#   h = MFGPU.analyze!(MFGPU.create(), A, S)
#   MFGPU.factor!(h, A, scale == SCALE_NONE ? nothing : Rs, check)
#   L, U, p, q, _ = MFGPU.factors(h; indextype = Ti)
#   return GPUPureLU(PureLU(L, U, p, q, Rs, A), h)
#
#   solve(F::GPUPureLU, b; refine=0) = MFGPU.solve(F.h, b; refine = refine)
#   Base.:\(F::GPUPureLU, b::AbstractVector) = solve(F, b)

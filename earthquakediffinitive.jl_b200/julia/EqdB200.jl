"""
    EqdB200

`ccall` binding of libeqd (include/eqd.h) for EarthquakeDiffinitive.jl.
It provides GPU versions of `fault_stiffness`, `fault_stiffness_toeplitz`,
`shear_traction` and the time-loop GEMV with the reference's argument
meaning and K layout (`Matrix{Float64}`, 2nf x 2nf, column-major).
It needs Julia on the host and a built `libeqd.so`; it does not depend on
the reference package.
"""
module EqdB200

using LinearAlgebra

export GpuFaultElasticity, gpu_fault_stiffness, gpu_fault_stiffness_toeplitz,
       gpu_shear_traction, GpuK, gpu_mul!, gpu_mul_device!, gpu_solver_report,
       GpuServer, serve!, submit, wait_request, request_info, GpuSplitNodeOperator

const libeqd = get(ENV, "EQD_LIB", joinpath(@__DIR__, "..", "lib", "libeqd.so"))

struct GridDesc
    n1::Int32; n2::Int32; n3::Int32
    x1_extent::Float64
    x2_lo::Float64; x2_hi::Float64; x3_lo::Float64; x3_hi::Float64
    lambda::Float64; mu::Float64; l_f::Float64
    order::Int32; device::Int32
end

# SolveOpts.flags bits (include/eqd.h)
const EQD_FLAG_STRICT = UInt32(1)    # return an error if a column did not converge
const EQD_FLAG_NO_SPLIT = UInt32(2)  # one chain of kernels instead of two overlapping halves
const EQD_FLAG_FUSE = UInt32(4)      # form the CG direction inside the stencil apply

mutable struct SolveOpts
    rtol::Float64; atol::Float64; itmax::Int64
    precond::Int32; precision::Int32; chunk::Int32
    reliable_delta::Float64; hbm_budget_bytes::UInt64
    variant::Int32; flags::UInt32
end

mutable struct Stats
    solves::Int64; iterations::Int64; max_iterations::Int64; unconverged::Int64
    reliable_updates::Int64; seconds::Float64; device_seconds::Float64
    precond::Int32; precision::Int32; kernel_launches::Int64
end
Stats() = Stats(0, 0, 0, 0, 0, 0.0, 0.0, 0, 0, 0)

function check(rc)
    rc == 0 && return nothing
    msg = unsafe_string(ccall((:eqd_last_error, libeqd), Cstring, ()))
    rc == 1 ? error(msg) : throw(ErrorException("libeqd error $rc: $msg"))
end

function default_opts(; rtol=1e-10, atol=0.0, itmax=0, precond=:none, precision=:mixed)
    o = SolveOpts(0, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    ccall((:eqd_default_opts, libeqd), Cvoid, (Ref{SolveOpts},), o)
    o.rtol, o.atol, o.itmax = rtol, atol, itmax
    precond in (:none, :jacobi) || error("precond must be :none or :jacobi, got $precond")
    o.precond = precond === :jacobi ? 1 : 0
    o.precision = precision === :fp64 ? 0 : 1
    return o
end

"""
    GpuFaultElasticity(n1, n23, L_fault, L_normal, λ, μ; l_f, device=0, solver_kwargs...)

The device-side analogue of `FaultElasticity` for `build_model`'s grids
(src/BP8.jl:196-206): minus block x1 ∈ [-L_normal, 0], plus block
x1 ∈ [0, L_normal], both x2, x3 ∈ [-L_fault, L_fault].
"""
mutable struct GpuFaultElasticity
    handle::Ptr{Cvoid}
    nf::Int
    n2f::Int
    n3f::Int
    opts::SolveOpts
    stats::Stats
end

function GpuFaultElasticity(n1, n23, L_fault, L_normal, λ, μ; l_f, device=0, solver_kwargs...)
    d = GridDesc(n1, n23, n23, L_normal, -L_fault, L_fault, -L_fault, L_fault, λ, μ, l_f, 4, device)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:eqd_grid_create, libeqd), Cint, (Ref{GridDesc}, Ref{Ptr{Cvoid}}), d, h))
    ntot = Ref{Int64}(0); nf = Ref{Int32}(0); n2f = Ref{Int32}(0); n3f = Ref{Int32}(0)
    check(ccall((:eqd_grid_info, libeqd), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int32}, Ref{Int32}, Ref{Int32}),
                h[], ntot, nf, n2f, n3f))
    fe = GpuFaultElasticity(h[], nf[], n2f[], n3f[], default_opts(; solver_kwargs...), Stats())
    finalizer(fe) do x
        x.handle == C_NULL || ccall((:eqd_grid_destroy, libeqd), Cint, (Ptr{Cvoid},), x.handle)
        x.handle = C_NULL
    end
    return fe
end

function merge!(fe::GpuFaultElasticity, st::Stats)
    t = fe.stats
    t.solves += st.solves; t.iterations += st.iterations
    t.max_iterations = max(t.max_iterations, st.max_iterations)
    t.unconverged += st.unconverged
    st.unconverged > 0 && @warn "CG did not converge on $(st.unconverged) split-node solve(s)"
    return fe
end

"`fault_stiffness(fe)` on the GPU (src/FaultResponse.jl:229-287)."
function gpu_fault_stiffness(fe::GpuFaultElasticity)
    K = Matrix{Float64}(undef, 2fe.nf, 2fe.nf)
    st = Stats()
    check(ccall((:eqd_stiffness_exact, libeqd), Cint, (Ptr{Cvoid}, Ref{SolveOpts}, Ptr{Float64}, Ref{Stats}),
                fe.handle, fe.opts, K, st))
    merge!(fe, st)
    return K
end

"`fault_stiffness_toeplitz(fe)` on the GPU (src/FaultResponse.jl:339-393)."
function gpu_fault_stiffness_toeplitz(fe::GpuFaultElasticity)
    K = Matrix{Float64}(undef, 2fe.nf, 2fe.nf)
    st = Stats()
    check(ccall((:eqd_stiffness_toeplitz, libeqd), Cint, (Ptr{Cvoid}, Ref{SolveOpts}, Ptr{Float64}, Ref{Stats}),
                fe.handle, fe.opts, K, st))
    merge!(fe, st)
    return K
end

"`shear_traction(fe, s2, s3)` on the GPU (src/FaultResponse.jl:194-211)."
function gpu_shear_traction(fe::GpuFaultElasticity, s2::AbstractVector, s3::AbstractVector)
    a2 = Vector{Float64}(s2); a3 = Vector{Float64}(s3)
    d2 = similar(a2); d3 = similar(a3)
    st = Stats()
    check(ccall((:eqd_shear_traction, libeqd), Cint,
                (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32, Ptr{Float64}, Ptr{Float64}, Ref{SolveOpts}, Ref{Stats}),
                fe.handle, a2, a3, 1, d2, d3, fe.opts, st))
    merge!(fe, st)
    return d2, d3
end

"`solver_report` (src/ElasticitySplitNode.jl:442-447)."
gpu_solver_report(fe::GpuFaultElasticity) =
    (; kind=:cg, precond=fe.opts.precond == 1 ? :jacobi : :none, solves=fe.stats.solves,
       iterations=fe.stats.iterations,
       mean_iterations=fe.stats.solves == 0 ? 0.0 : fe.stats.iterations / fe.stats.solves,
       max_iterations=fe.stats.max_iterations, unconverged=fe.stats.unconverged)

"""
    GpuSplitNodeOperator(fe; mode=:A, precision=:fp64)

The split-node operator as a matrix-free linear map on the GPU, for callers
that want `A` or `HP_DSAT` (src/ElasticitySplitNode.jl:210-211) without
assembling them: `mul!(y, op, x)` applies `A = -HP(D+SAT)P` (`mode=:A`) or
`HP(D+SAT)` (`mode=:HP_DSAT`) to vectors in the reference DOF layout, so
Krylov.jl on the host can drive the GPU stencil.
"""
struct GpuSplitNodeOperator
    fe::GpuFaultElasticity
    mode::Int32
    precision::Int32
    n::Int
end

function GpuSplitNodeOperator(fe::GpuFaultElasticity; mode=:A, precision=:fp64)
    ntot = Ref{Int64}(0); nf = Ref{Int32}(0); n2f = Ref{Int32}(0); n3f = Ref{Int32}(0)
    check(ccall((:eqd_grid_info, libeqd), Cint, (Ptr{Cvoid}, Ref{Int64}, Ref{Int32}, Ref{Int32}, Ref{Int32}),
                fe.handle, ntot, nf, n2f, n3f))
    mode in (:A, :HP_DSAT) || error("mode must be :A or :HP_DSAT, got $mode")
    return GpuSplitNodeOperator(fe, mode === :A ? 0 : 1, precision === :fp64 ? 0 : 1, Int(ntot[]))
end

Base.size(op::GpuSplitNodeOperator) = (op.n, op.n)
Base.size(op::GpuSplitNodeOperator, d::Integer) = d <= 2 ? op.n : 1
Base.eltype(::GpuSplitNodeOperator) = Float64

function LinearAlgebra.mul!(y::AbstractVecOrMat{Float64}, op::GpuSplitNodeOperator, x::AbstractVecOrMat{Float64})
    size(x, 1) == op.n && size(y) == size(x) || throw(DimensionMismatch("operator is $(op.n) x $(op.n)"))
    xc = Matrix{Float64}(reshape(x, op.n, :)); yc = similar(xc)
    check(ccall((:eqd_apply, libeqd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32, Int32, Int32),
                op.fe.handle, xc, yc, size(xc, 2), op.mode, op.precision))
    copyto!(y, yc)
    return y
end

"K resident on the device for the time loop's `mul!(Δτ, K, slip)` (src/BP8.jl:366)."
mutable struct GpuK
    handle::Ptr{Cvoid}
    n::Int
end

function GpuK(K::Matrix{Float64}; device=0)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:eqd_kmat_create, libeqd), Cint, (Int32, Int32, Ptr{Float64}, Ref{Ptr{Cvoid}}),
                device, size(K, 1), K, h))
    g = GpuK(h[], size(K, 1))
    finalizer(g) do x
        x.handle == C_NULL || ccall((:eqd_kmat_destroy, libeqd), Cint, (Ptr{Cvoid},), x.handle)
        x.handle = C_NULL
    end
    return g
end

function gpu_mul!(y::Vector{Float64}, K::GpuK, s::Vector{Float64})
    check(ccall((:eqd_kmat_gemv, libeqd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32),
                K.handle, s, y, 1))
    return y
end

"`Y = K S` for the columns of `S` (n x nvec; from 3 columns on, on the FP64 tensor cores)."
function gpu_mul!(Y::Matrix{Float64}, K::GpuK, S::Matrix{Float64})
    size(S, 1) == K.n && size(Y) == size(S) || throw(DimensionMismatch("K is $(K.n) x $(K.n), S $(size(S)), Y $(size(Y))"))
    check(ccall((:eqd_kmat_gemv, libeqd), Cint, (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Int32),
                K.handle, S, Y, size(S, 2)))
    return Y
end

"""
    gpu_mul_device!(y_ptr, K, s_ptr, nvec; stream=C_NULL)

`y = K s` on slip vectors already on the device (e.g. `pointer(s)` of a
`CuMatrix{Float64}` of n x nvec, column-major), launched on `stream` (a
`CUstream` handle) without a synchronize. Calls on one `GpuK` must be
serialised; the first call of a size may allocate scratch (make it before
stream capture).
"""
function gpu_mul_device!(y_ptr, K::GpuK, s_ptr, nvec::Integer; stream=C_NULL)
    check(ccall((:eqd_kmat_gemv_device, libeqd), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Cvoid}, Int32, Ptr{Cvoid}),
                K.handle, Ptr{Cvoid}(UInt(s_ptr)), Ptr{Cvoid}(UInt(y_ptr)), nvec, Ptr{Cvoid}(UInt(stream))))
    return y_ptr
end

# ---------------------------------------------------------------------------
# Request serving (eqd_server_*): continuous batching of K-column requests
# ---------------------------------------------------------------------------
struct RequestInfo
    state::Int32; ncols::Int32; unconverged::Int32; max_iterations::Int32
    iterations::Int64; t_submit::Float64; t_start::Float64; t_done::Float64
end

mutable struct GpuServer
    handle::Ptr{Cvoid}
    outputs::Dict{Int64,Matrix{Float64}}   # keeps each request's K buffer alive
end

function GpuServer(; hbm_budget_bytes=150_000_000_000, solver_kwargs...)
    o = default_opts(; solver_kwargs...)
    h = Ref{Ptr{Cvoid}}(C_NULL)
    check(ccall((:eqd_server_create, libeqd), Cint, (Ref{SolveOpts}, UInt64, Ref{Ptr{Cvoid}}),
                o, UInt64(hbm_budget_bytes), h))
    s = GpuServer(h[], Dict{Int64,Matrix{Float64}}())
    finalizer(s) do x
        x.handle == C_NULL || ccall((:eqd_server_destroy, libeqd), Cint, (Ptr{Cvoid},), x.handle)
        x.handle = C_NULL
    end
    return s
end

"Attach a grid (it belongs to the server from now on); `slots = 0` sizes the slot pool from the budget."
serve!(s::GpuServer, fe::GpuFaultElasticity; slots=0) =
    check(ccall((:eqd_server_add_grid, libeqd), Cint, (Ptr{Cvoid}, Ptr{Cvoid}, Int32), s.handle, fe.handle, slots))

"Queue K columns `cols` (1-based, as K's column indices) of an attached grid; returns the request id."
function submit(s::GpuServer, fe::GpuFaultElasticity, cols::AbstractVector{<:Integer})
    out = Matrix{Float64}(undef, 2fe.nf, length(cols))
    id = Ref{Int64}(0)
    c = Int32.(cols .- 1)
    check(ccall((:eqd_server_submit, libeqd), Cint,
                (Ptr{Cvoid}, Ptr{Cvoid}, Ptr{Int32}, Int32, Ptr{Float64}, Ref{Int64}),
                s.handle, fe.handle, c, length(c), out, id))
    s.outputs[id[]] = out
    return id[]
end

"Block until the request is done; returns its K columns (2nf x length(cols))."
function wait_request(s::GpuServer, id::Int64; timeout=-1.0)
    check(ccall((:eqd_server_wait, libeqd), Cint, (Ptr{Cvoid}, Int64, Float64), s.handle, id, timeout))
    return s.outputs[id]
end

function request_info(s::GpuServer, id::Int64)
    r = Ref{RequestInfo}()
    check(ccall((:eqd_server_request_info, libeqd), Cint, (Ptr{Cvoid}, Int64, Ref{RequestInfo}), s.handle, id, r))
    return r[]
end

end # module

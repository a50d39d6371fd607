"""
    CompasToolkit

Julia interface to `libcompas_b200.so`, the B200 (sm_100a) library of the COMPAS simulation hot path
(FISP / pSSFP Bloch simulation, Cartesian and spiral signal, Jacobian products, residual).

The functions, constructors and keyword arguments have the names, argument order and array shapes of
the reference's `CompasToolkit.jl` module, so code written against that module runs unchanged:

  * arrays are Julia column-major: echos are `nvoxels × nreadouts`, coil sensitivities
    `nvoxels × ncoils`, signals `samples × nreadouts × ncoils`, Jᴴ·v results `nvoxels × 4`;
  * inputs may be host arrays (converted to `Float32` / `ComplexF32` and uploaded) or `CompasArray`s
    already on the device (used as they are);
  * results are `CompasArray`s that stay on the device until `collect` copies them back.

Differences from the reference module:

  * `pSSFPSequence` passes the slice positions `z` as `Float32`, the type the library reads (the
    reference module converts them to `ComplexF32`);
  * a failing call raises `ErrorException` with the library's message (`compas_last_error`);
  * `simulate_magnetization_tangents` returns m, ∂m/∂T1 and ∂m/∂T2 of one pass (exact forward-mode
    derivatives) in place of a simulation plus two finite differences;
  * `low_precision = true` and `false` both run the split-BF16 tensor-core products (relative error
    ≤ 1e-4 against FP64).

`Constants.jl` (written by `make -C compas-toolkit_b200 julia`) defines `LIBRARY`, the path of the
library, and `VERSION`, the version string it must report.
"""
module CompasToolkit

include("Constants.jl")

using Base.ScopedValues

"""
    LOW_PRECISION_MODE

Default of the `low_precision` keyword of the signal and Jacobian functions; set it for a scope
with `with(CompasToolkit.LOW_PRECISION_MODE => true) do ... end`.
"""
const LOW_PRECISION_MODE = ScopedValue(false)

const CONTEXT_KEY = :compas_b200_context

# ------------------------------------------------------------------------------------------------
# errors, version
# ------------------------------------------------------------------------------------------------

"""Raise the library's message for the failed call `what` when `ptr` is NULL; else return `ptr`."""
function checked(ptr::Ptr{Cvoid}, what::AbstractString)::Ptr{Cvoid}
    if ptr == C_NULL
        msg = @ccall LIBRARY.compas_last_error()::Cstring
        detail = msg == C_NULL ? "failed" : unsafe_string(msg)
        throw(ErrorException("$what: $detail"))
    end
    return ptr
end

"""Raise the library's message when the call that just returned reported an error."""
function check_last_error(what::AbstractString)
    msg = @ccall LIBRARY.compas_last_error()::Cstring
    msg == C_NULL || throw(ErrorException("$what: $(unsafe_string(msg))"))
    return nothing
end

"""
    version()::String

Version string of the loaded library.
"""
version()::String = unsafe_string(@ccall LIBRARY.compas_version()::Cstring)

"""
    check_version()

Raise an error when the loaded library is not the version `Constants.jl` names.
"""
function check_version()
    got = version()
    got == VERSION || throw(ErrorException("`$LIBRARY` reports version $got; this module expects $VERSION"))
    return nothing
end

# ------------------------------------------------------------------------------------------------
# handles
# ------------------------------------------------------------------------------------------------

"""Objects that own one library handle in a field `ptr`; `@ccall` arguments of type
`Ptr{Cvoid}` accept them directly (the object stays rooted for the call)."""
abstract type Handle end

Base.unsafe_convert(::Type{Ptr{Cvoid}}, h::Handle) = h.ptr
Base.pointer(h::Handle) = h.ptr

destroy_object(h::Handle) = @ccall LIBRARY.compas_destroy_object(h.ptr::Ptr{Cvoid})::Cvoid

"""
    Context()
    Context(context::Context, device::Integer)

A library context: one device and one CUDA stream on which all its work is ordered. The second form
copies `context` for another device.
"""
mutable struct Context <: Handle
    ptr::Ptr{Cvoid}

    function Context(ptr::Ptr{Cvoid})
        ctx = new(checked(ptr, "compas_make_context"))
        return finalizer(ctx) do c
            @ccall LIBRARY.compas_destroy_context(c.ptr::Ptr{Cvoid})::Cvoid
        end
    end
end

function Context()
    check_version()
    return Context(@ccall LIBRARY.compas_make_context()::Ptr{Cvoid})
end

function Context(context::Context, device::Integer)
    check_version()
    return Context(@ccall LIBRARY.compas_copy_context_for_device(context::Ptr{Cvoid}, device::Int32)::Ptr{Cvoid})
end

Base.show(io::IO, ::Context) = print(io, "Context()")

"""
    set_context(context::Context)
    set_context(context::Context, device::Integer)

Make `context` (or its copy for `device`) the context of the current task.
"""
set_context(context::Context) = task_local_storage(CONTEXT_KEY, context)
set_context(context::Context, device::Integer) = task_local_storage(CONTEXT_KEY, Context(context, device))

"""
    get_context()::Context

The current task's context; an error when `init_context` / `set_context` has not been called.
"""
function get_context()::Context
    ctx = get(task_local_storage(), CONTEXT_KEY, nothing)
    ctx === nothing && throw(ArgumentError("no COMPAS context: call `CompasToolkit.init_context()` first"))
    return ctx
end

"""
    init_context(device::Integer=0)::Context

Create a context on `device`, make it the current task's context and return it.
"""
function init_context(device::Integer=0)::Context
    set_context(Context(), device)
    return get_context()
end

"""
    synchronize()

Wait until the current context's queued work has finished.
"""
function synchronize()
    @ccall LIBRARY.compas_synchronize(get_context()::Ptr{Cvoid})::Cvoid
    check_last_error("compas_synchronize")
end

# ------------------------------------------------------------------------------------------------
# device arrays
# ------------------------------------------------------------------------------------------------

"""
    CompasArray{T, N} <: AbstractArray{T, N}

An `N`-dimensional array of `T` (`Float32` or `ComplexF32`) in device memory. Indexing is not
supported; `collect` copies it to the host.
"""
mutable struct CompasArray{T, N} <: AbstractArray{T, N}
    context::Context
    ptr::Ptr{Cvoid}
    extents::Dims{N}  # the library's extents, slowest axis first (the reverse of `size`)

    function CompasArray{T, N}(context::Context, ptr::Ptr{Cvoid}, extents::Dims{N}) where {T, N}
        a = new{T, N}(context, checked(ptr, "compas array"), extents)
        return finalizer(a) do x
            @ccall LIBRARY.compas_destroy_array(x.ptr::Ptr{Cvoid})::Cvoid
        end
    end
end

Base.size(a::CompasArray) = reverse(a.extents)
Base.getindex(::CompasArray, i...) = throw(ArgumentError("a CompasArray lives on the device: `collect` it first"))
Base.unsafe_convert(::Type{Ptr{Cvoid}}, a::CompasArray) = a.ptr
Base.pointer(a::CompasArray) = a.ptr
Base.show(io::IO, a::CompasArray) = print(io, typeof(a), " of size ", size(a))
Base.show(io::IO, ::MIME"text/plain", a::CompasArray) = show(io, a)

extents_of(x::AbstractArray) = Int64[reverse(size(x))...]

function CompasArray(host::Array{Float32, N}) where {N}
    ctx = get_context()
    ext = extents_of(host)
    ptr = @ccall LIBRARY.compas_make_array_float(ctx::Ptr{Cvoid}, host::Ptr{Float32}, N::Int32,
                                                 ext::Ptr{Int64})::Ptr{Cvoid}
    return CompasArray{Float32, N}(ctx, checked(ptr, "compas_make_array_float"), Dims{N}(ext))
end

function CompasArray(host::Array{ComplexF32, N}) where {N}
    ctx = get_context()
    ext = extents_of(host)
    ptr = @ccall LIBRARY.compas_make_array_complex(ctx::Ptr{Cvoid}, host::Ptr{ComplexF32}, N::Int32,
                                                   ext::Ptr{Int64})::Ptr{Cvoid}
    return CompasArray{ComplexF32, N}(ctx, checked(ptr, "compas_make_array_complex"), Dims{N}(ext))
end

function Base.collect(a::CompasArray{Float32, N}) where {N}
    out = Array{Float32, N}(undef, size(a))
    @ccall LIBRARY.compas_read_array_float(a.context::Ptr{Cvoid}, a::Ptr{Cvoid}, out::Ptr{Float32},
                                           length(out)::Int64)::Cvoid
    check_last_error("compas_read_array_float")
    return out
end

function Base.collect(a::CompasArray{ComplexF32, N}) where {N}
    out = Array{ComplexF32, N}(undef, size(a))
    @ccall LIBRARY.compas_read_array_complex(a.context::Ptr{Cvoid}, a::Ptr{Cvoid}, out::Ptr{ComplexF32},
                                             length(out)::Int64)::Cvoid
    check_last_error("compas_read_array_complex")
    return out
end

function check_size(x::AbstractArray, dims::Dims)
    size(x) == dims || throw(ArgumentError("array of size $(size(x)) where $dims is required"))
    return nothing
end

"""Device array of element type `T` and Julia size `dims`: a matching `CompasArray` as it is, any
other array converted and uploaded."""
function device_array(x::CompasArray, ::Type{T}, dims::Integer...) where {T}
    eltype(x) === T || throw(ArgumentError("a CompasArray of $T is required, got one of $(eltype(x))"))
    check_size(x, Dims(dims))
    return x
end

function device_array(x::AbstractArray, ::Type{T}, dims::Integer...) where {T}
    check_size(x, Dims(dims))
    return CompasArray(convert(Array{T, length(dims)}, x))
end

"""Host vector of `n` `Float32`: a number repeated, or a vector of length `n` converted."""
host_vector(x::Number, n::Integer) = fill(Float32(x), n)

function host_vector(x::AbstractVector, n::Integer)
    check_size(x, (Int(n),))
    return convert(Vector{Float32}, x)
end

# ------------------------------------------------------------------------------------------------
# tissue, sequences, trajectories
# ------------------------------------------------------------------------------------------------

"""
    TissueParameters(nvoxels, T1, T2, B1, B0, rho_x, rho_y, x, y[, z])

Per-voxel parameters (vectors of `nvoxels`, or numbers repeated for every voxel); `z` defaults to 0.
"""
mutable struct TissueParameters <: Handle
    ptr::Ptr{Cvoid}
    nvoxels::Int32

    function TissueParameters(nvoxels::Integer, T1, T2, B1, B0, rho_x, rho_y, x, y, z=0.0f0)
        ctx = get_context()
        f = [host_vector(v, nvoxels) for v in (T1, T2, B1, B0, rho_x, rho_y, x, y, z)]
        ptr = @ccall LIBRARY.compas_make_tissue_parameters(
            ctx::Ptr{Cvoid}, nvoxels::Int32, f[1]::Ptr{Float32}, f[2]::Ptr{Float32}, f[3]::Ptr{Float32},
            f[4]::Ptr{Float32}, f[5]::Ptr{Float32}, f[6]::Ptr{Float32}, f[7]::Ptr{Float32}, f[8]::Ptr{Float32},
            f[9]::Ptr{Float32})::Ptr{Cvoid}
        return finalizer(destroy_object, new(checked(ptr, "compas_make_tissue_parameters"), nvoxels))
    end
end

Base.show(io::IO, p::TissueParameters) = print(io, "TissueParameters(nvoxels=$(p.nvoxels))")

"""
    FispSequence(RF_train, slice_profiles, TR, TE, max_state, TI; undersampling_factor=1, repetitions=1)

FISP sequence: `RF_train` (nTR complex flip angles in degrees), `slice_profiles` (nTR × positions),
TR / TE / TI in seconds and `max_state` EPG states; the echo count is nTR × `undersampling_factor`.
"""
mutable struct FispSequence <: Handle
    ptr::Ptr{Cvoid}
    nreadouts::Int32

    function FispSequence(RF_train::AbstractVector, slice_profiles::AbstractMatrix, TR::Number, TE::Number,
                          max_state::Integer, TI::Number; undersampling_factor::Number=1, repetitions::Number=1)
        ntr = length(RF_train)
        rf = device_array(RF_train, ComplexF32, ntr)
        profiles = device_array(slice_profiles, ComplexF32, ntr, size(slice_profiles, 2))
        TW = 0.0f0  # the module's sequences have no wait time before the inversion
        ptr = @ccall LIBRARY.compas_make_fisp_sequence(
            rf::Ptr{Cvoid}, profiles::Ptr{Cvoid}, TR::Float32, TE::Float32, TW::Float32, max_state::Int32,
            TI::Float32, undersampling_factor::Int32, repetitions::Int32)::Ptr{Cvoid}
        return finalizer(destroy_object, new(checked(ptr, "compas_make_fisp_sequence"),
                                             ntr * undersampling_factor))
    end
end

"""
    pSSFPSequence(RF_train, TR, gamma_dt_RF, dt, gamma_dt_GRz, z)

pSSFP sequence: `RF_train` (nTR complex), TR, the RF waveform `gamma_dt_RF`, the (excitation,
inversion, preparation) time steps `dt` and gradient steps `gamma_dt_GRz`, and the slice positions
`z` (real).
"""
mutable struct pSSFPSequence <: Handle
    ptr::Ptr{Cvoid}
    nreadouts::Int32

    function pSSFPSequence(RF_train::AbstractVector, TR::AbstractFloat, gamma_dt_RF::AbstractVector,
                           dt::NTuple{3, <:AbstractFloat}, gamma_dt_GRz::NTuple{3, <:AbstractFloat},
                           z::AbstractVector)
        ntr = length(RF_train)
        rf = device_array(RF_train, ComplexF32, ntr)
        wave = device_array(gamma_dt_RF, ComplexF32, length(gamma_dt_RF))
        zpos = device_array(z, Float32, length(z))
        ptr = @ccall LIBRARY.compas_make_pssfp_sequence(
            rf::Ptr{Cvoid}, TR::Float32, wave::Ptr{Cvoid}, dt[1]::Float32, dt[2]::Float32, dt[3]::Float32,
            gamma_dt_GRz[1]::Float32, gamma_dt_GRz[2]::Float32, gamma_dt_GRz[3]::Float32,
            zpos::Ptr{Cvoid})::Ptr{Cvoid}
        return finalizer(destroy_object, new(checked(ptr, "compas_make_pssfp_sequence"), ntr))
    end
end

"""Readout trajectories: `CartesianTrajectory` and `SpiralTrajectory`."""
abstract type Trajectory <: Handle end

"""
    CartesianTrajectory(nreadouts, samples_per_readout, delta_t, k_start, delta_k)

Cartesian readouts: readout r starts at `k_start[r]` and moves by the real step `delta_k` per sample.
"""
mutable struct CartesianTrajectory <: Trajectory
    ptr::Ptr{Cvoid}
    nreadouts::Int32
    samples_per_readout::Int32

    function CartesianTrajectory(nreadouts::Integer, samples_per_readout::Integer, delta_t::Number,
                                 k_start::AbstractVector, delta_k::Number)
        ks = device_array(k_start, ComplexF32, nreadouts)
        ptr = @ccall LIBRARY.compas_make_cartesian_trajectory(
            nreadouts::Int32, samples_per_readout::Int32, delta_t::Float32, ks::Ptr{Cvoid},
            delta_k::Float32)::Ptr{Cvoid}
        return finalizer(destroy_object, new(checked(ptr, "compas_make_cartesian_trajectory"), nreadouts,
                                             samples_per_readout))
    end
end

"""
    SpiralTrajectory(nreadouts, samples_per_readout, delta_t, k_start, delta_k)

Spiral readouts: readout r starts at `k_start[r]` and moves by the complex step `delta_k[r]` per
sample.
"""
mutable struct SpiralTrajectory <: Trajectory
    ptr::Ptr{Cvoid}
    nreadouts::Int32
    samples_per_readout::Int32

    function SpiralTrajectory(nreadouts::Integer, samples_per_readout::Integer, delta_t::Number,
                              k_start::AbstractVector, delta_k::AbstractVector)
        ks = device_array(k_start, ComplexF32, nreadouts)
        dk = device_array(delta_k, ComplexF32, nreadouts)
        ptr = @ccall LIBRARY.compas_make_spiral_trajectory(
            nreadouts::Int32, samples_per_readout::Int32, delta_t::Float32, ks::Ptr{Cvoid},
            dk::Ptr{Cvoid})::Ptr{Cvoid}
        return finalizer(destroy_object, new(checked(ptr, "compas_make_spiral_trajectory"), nreadouts,
                                             samples_per_readout))
    end
end

function Base.show(io::IO, t::Trajectory)
    print(io, nameof(typeof(t)), "(nreadouts=$(t.nreadouts), samples_per_readout=$(t.samples_per_readout))")
end

# ------------------------------------------------------------------------------------------------
# simulation
# ------------------------------------------------------------------------------------------------

echo_array(ctx::Context, ptr::Ptr{Cvoid}, p::TissueParameters, seq) =
    CompasArray{ComplexF32, 2}(ctx, ptr, (Int(seq.nreadouts), Int(p.nvoxels)))

"""
    simulate_magnetization(parameters, sequence)::CompasArray{ComplexF32, 2}

Transverse magnetization at the echo times, `nvoxels × nreadouts`, for a `FispSequence` or a
`pSSFPSequence`.
"""
function simulate_magnetization(parameters::TissueParameters, sequence::FispSequence)
    ctx = get_context()
    ptr = @ccall LIBRARY.compas_simulate_magnetization_fisp(ctx::Ptr{Cvoid}, parameters::Ptr{Cvoid},
                                                            sequence::Ptr{Cvoid})::Ptr{Cvoid}
    return echo_array(ctx, checked(ptr, "compas_simulate_magnetization_fisp"), parameters, sequence)
end

function simulate_magnetization(parameters::TissueParameters, sequence::pSSFPSequence)
    ctx = get_context()
    ptr = @ccall LIBRARY.compas_simulate_magnetization_pssfp(ctx::Ptr{Cvoid}, parameters::Ptr{Cvoid},
                                                             sequence::Ptr{Cvoid})::Ptr{Cvoid}
    return echo_array(ctx, checked(ptr, "compas_simulate_magnetization_pssfp"), parameters, sequence)
end

"""
    simulate_magnetization_derivative(field, echos, parameters, sequence, Δ)::CompasArray{ComplexF32, 2}

Forward difference (m(p + Δ·p[field]) − m) / (Δ·p[field]) of the echos with respect to tissue field
`field` (0 = T1, 1 = T2, ...), given the unperturbed `echos` (`nvoxels × nreadouts`).
"""
function simulate_magnetization_derivative(field::Integer, echos::AbstractMatrix, parameters::TissueParameters,
                                           sequence::FispSequence, Δ::AbstractFloat)
    ctx = get_context()
    e = device_array(echos, ComplexF32, parameters.nvoxels, sequence.nreadouts)
    ptr = @ccall LIBRARY.compas_simulate_magnetization_derivative_fisp(
        ctx::Ptr{Cvoid}, field::Int32, e::Ptr{Cvoid}, parameters::Ptr{Cvoid}, Δ::Float32,
        sequence::Ptr{Cvoid})::Ptr{Cvoid}
    return echo_array(ctx, checked(ptr, "compas_simulate_magnetization_derivative_fisp"), parameters, sequence)
end

function simulate_magnetization_derivative(field::Integer, echos::AbstractMatrix, parameters::TissueParameters,
                                           sequence::pSSFPSequence, Δ::AbstractFloat)
    ctx = get_context()
    e = device_array(echos, ComplexF32, parameters.nvoxels, sequence.nreadouts)
    ptr = @ccall LIBRARY.compas_simulate_magnetization_derivative_pssfp(
        ctx::Ptr{Cvoid}, field::Int32, e::Ptr{Cvoid}, parameters::Ptr{Cvoid}, Δ::Float32,
        sequence::Ptr{Cvoid})::Ptr{Cvoid}
    return echo_array(ctx, checked(ptr, "compas_simulate_magnetization_derivative_pssfp"), parameters, sequence)
end

"""
    simulate_magnetization_derivatives(echos, parameters, sequence[, Δ = 1e-4])

`(T1 = ∂m/∂T1, T2 = ∂m/∂T2)` by forward differences of relative step Δ.
"""
function simulate_magnetization_derivatives(echos::AbstractMatrix, parameters::TissueParameters, sequence,
                                            Δ::AbstractFloat=1e-4)
    return (T1 = simulate_magnetization_derivative(0, echos, parameters, sequence, Δ),
            T2 = simulate_magnetization_derivative(1, echos, parameters, sequence, Δ))
end

"""
    simulate_magnetization_tangents(parameters, sequence)

`(echos, (T1 = ∂m/∂T1, T2 = ∂m/∂T2))` from one simulation that carries the exact derivatives with
the state (forward mode), for a `FispSequence` or a `pSSFPSequence`.
"""
function simulate_magnetization_tangents(parameters::TissueParameters, sequence::Union{FispSequence, pSSFPSequence})
    ctx = get_context()
    m, dT1, dT2 = Ref(C_NULL), Ref(C_NULL), Ref(C_NULL)
    rc = @ccall LIBRARY.compas_b200_simulate_magnetization_tangents(
        ctx::Ptr{Cvoid}, parameters::Ptr{Cvoid}, sequence::Ptr{Cvoid}, m::Ptr{Ptr{Cvoid}}, dT1::Ptr{Ptr{Cvoid}},
        dT2::Ptr{Ptr{Cvoid}})::Cint
    rc == 0 || checked(C_NULL, "compas_b200_simulate_magnetization_tangents")
    echos = echo_array(ctx, m[], parameters, sequence)
    return echos, (T1 = echo_array(ctx, dT1[], parameters, sequence), T2 = echo_array(ctx, dT2[], parameters, sequence))
end

# ------------------------------------------------------------------------------------------------
# signal, Jacobian products, phase encoding, residual
# ------------------------------------------------------------------------------------------------

signal_array(ctx::Context, ptr::Ptr{Cvoid}, ncoils, t::Trajectory) =
    CompasArray{ComplexF32, 3}(ctx, ptr, (Int(ncoils), Int(t.nreadouts), Int(t.samples_per_readout)))

"""
    magnetization_to_signal(echos, parameters, trajectory, coils; low_precision)::CompasArray{ComplexF32, 3}

Signal `samples × nreadouts × ncoils` of the echos (`nvoxels × nreadouts`) received through the coil
sensitivities (`nvoxels × ncoils`) along a Cartesian or spiral trajectory.
"""
function magnetization_to_signal(echos::AbstractMatrix, parameters::TissueParameters,
                                 trajectory::CartesianTrajectory, coils::AbstractMatrix;
                                 low_precision::Bool=LOW_PRECISION_MODE[])
    ctx = get_context()
    nv, nc = Int(parameters.nvoxels), size(coils, 2)
    e = device_array(echos, ComplexF32, nv, trajectory.nreadouts)
    c = device_array(coils, ComplexF32, nv, nc)
    ptr = @ccall LIBRARY.compas_magnetization_to_signal_cartesian(
        ctx::Ptr{Cvoid}, nc::Int32, e::Ptr{Cvoid}, parameters::Ptr{Cvoid}, c::Ptr{Cvoid},
        trajectory::Ptr{Cvoid}, low_precision::Int32)::Ptr{Cvoid}
    return signal_array(ctx, checked(ptr, "compas_magnetization_to_signal_cartesian"), nc, trajectory)
end

function magnetization_to_signal(echos::AbstractMatrix, parameters::TissueParameters,
                                 trajectory::SpiralTrajectory, coils::AbstractMatrix;
                                 low_precision::Bool=LOW_PRECISION_MODE[])
    ctx = get_context()
    nv, nc = Int(parameters.nvoxels), size(coils, 2)
    e = device_array(echos, ComplexF32, nv, trajectory.nreadouts)
    c = device_array(coils, ComplexF32, nv, nc)
    ptr = @ccall LIBRARY.compas_magnetization_to_signal_spiral(
        ctx::Ptr{Cvoid}, nc::Int32, e::Ptr{Cvoid}, parameters::Ptr{Cvoid}, c::Ptr{Cvoid},
        trajectory::Ptr{Cvoid})::Ptr{Cvoid}
    return signal_array(ctx, checked(ptr, "compas_magnetization_to_signal_spiral"), nc, trajectory)
end

"""
    compute_jacobian(echos, ∂echos, parameters, trajectory, coils, v; low_precision)::CompasArray{ComplexF32, 3}

J·v: the signal's directional derivative along `v` (`nvoxels × 4`: T1, T2, ρx, ρy per voxel), given
the echos and `∂echos = (T1 = ..., T2 = ...)` (each `nvoxels × nreadouts`); `samples × nreadouts × ncoils`.
"""
function compute_jacobian(echos::AbstractMatrix, ∂echos::NamedTuple{(:T1, :T2)}, parameters::TissueParameters,
                          trajectory::Trajectory, coils::AbstractMatrix, v::AbstractMatrix;
                          low_precision::Bool=LOW_PRECISION_MODE[])
    ctx = get_context()
    nv, nr, nc = Int(parameters.nvoxels), Int(trajectory.nreadouts), size(coils, 2)
    e = device_array(echos, ComplexF32, nv, nr)
    d1 = device_array(∂echos.T1, ComplexF32, nv, nr)
    d2 = device_array(∂echos.T2, ComplexF32, nv, nr)
    c = device_array(coils, ComplexF32, nv, nc)
    vec = device_array(v, ComplexF32, nv, 4)
    ptr = @ccall LIBRARY.compas_compute_jacobian(
        ctx::Ptr{Cvoid}, nc::Int32, e::Ptr{Cvoid}, d1::Ptr{Cvoid}, d2::Ptr{Cvoid}, parameters::Ptr{Cvoid},
        c::Ptr{Cvoid}, trajectory::Ptr{Cvoid}, vec::Ptr{Cvoid}, low_precision::Int32)::Ptr{Cvoid}
    return signal_array(ctx, checked(ptr, "compas_compute_jacobian"), nc, trajectory)
end

"""
    compute_jacobian_hermitian(echos, ∂echos, parameters, trajectory, coils, v; low_precision)::CompasArray{ComplexF32, 2}

Jᴴ·v of a signal-shaped `v` (`samples × nreadouts × ncoils`): `nvoxels × 4` (T1, T2, ρx, ρy).
"""
function compute_jacobian_hermitian(echos::AbstractMatrix, ∂echos::NamedTuple{(:T1, :T2)},
                                    parameters::TissueParameters, trajectory::Trajectory, coils::AbstractMatrix,
                                    v::AbstractArray{<:Any, 3}; low_precision::Bool=LOW_PRECISION_MODE[])
    ctx = get_context()
    nv, nr, nc = Int(parameters.nvoxels), Int(trajectory.nreadouts), size(coils, 2)
    e = device_array(echos, ComplexF32, nv, nr)
    d1 = device_array(∂echos.T1, ComplexF32, nv, nr)
    d2 = device_array(∂echos.T2, ComplexF32, nv, nr)
    c = device_array(coils, ComplexF32, nv, nc)
    vec = device_array(v, ComplexF32, trajectory.samples_per_readout, nr, nc)
    ptr = @ccall LIBRARY.compas_compute_jacobian_hermitian(
        ctx::Ptr{Cvoid}, nc::Int32, e::Ptr{Cvoid}, d1::Ptr{Cvoid}, d2::Ptr{Cvoid}, parameters::Ptr{Cvoid},
        trajectory::Ptr{Cvoid}, c::Ptr{Cvoid}, vec::Ptr{Cvoid}, low_precision::Int32)::Ptr{Cvoid}
    return CompasArray{ComplexF32, 2}(ctx, checked(ptr, "compas_compute_jacobian_hermitian"), (4, nv))
end

"""
    phase_encoding(echos, parameters, trajectory)::CompasArray{ComplexF32, 2}
    phase_encoding(inputs::NamedTuple, parameters, trajectory)::NamedTuple

Echos multiplied by each voxel's phase at the start of every readout (`nvoxels × nreadouts`); the
second form applies it to every array of a named tuple.
"""
function phase_encoding(echos::AbstractMatrix, parameters::TissueParameters, trajectory::Trajectory)
    ctx = get_context()
    e = device_array(echos, ComplexF32, parameters.nvoxels, trajectory.nreadouts)
    ptr = @ccall LIBRARY.phase_encoding(ctx::Ptr{Cvoid}, e::Ptr{Cvoid}, parameters::Ptr{Cvoid},
                                        trajectory::Ptr{Cvoid})::Ptr{Cvoid}
    return CompasArray{ComplexF32, 2}(ctx, checked(ptr, "phase_encoding"),
                                      (Int(trajectory.nreadouts), Int(parameters.nvoxels)))
end

phase_encoding(inputs::NamedTuple, parameters::TissueParameters, trajectory::Trajectory) =
    map(x -> phase_encoding(x, parameters, trajectory), inputs)

"""
    compute_residual(lhs, rhs)::Tuple{Float32, CompasArray{ComplexF32, 3}}

`(Σ|lhs − rhs|², lhs − rhs)` of two arrays of the same three-dimensional size.
"""
function compute_residual(lhs::AbstractArray{<:Any, 3}, rhs::AbstractArray{<:Any, 3})
    ctx = get_context()
    dims = size(lhs)
    a = device_array(lhs, ComplexF32, dims...)
    b = device_array(rhs, ComplexF32, dims...)
    objective = Ref{Float32}(0)
    ptr = @ccall LIBRARY.compas_compute_residual(ctx::Ptr{Cvoid}, a::Ptr{Cvoid}, b::Ptr{Cvoid},
                                                 objective::Ptr{Float32})::Ptr{Cvoid}
    diff = CompasArray{ComplexF32, 3}(ctx, checked(ptr, "compas_compute_residual"), reverse(dims))
    return objective[], diff
end

end  # module CompasToolkit

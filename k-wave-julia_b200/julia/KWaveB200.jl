"""
    KWaveB200

Runs KWave.jl's k-space time stepping (fluid, axisymmetric and elastic solvers) on an NVIDIA B200 through libkwb's C ABI
(`include/kwb.h`).  `KWaveB200.kspace_first_order` has the signature and output of
`KWave.kspace_first_order` (KWave.jl/src/solver/first_order.jl:92-111, 287-306, 505-524):

    using KWave, KWaveB200
    out = KWaveB200.kspace_first_order(kgrid, medium, source, sensor; pml_size=20, smooth_p0=true)

or, to switch every call site at once, `import KWaveB200: kspace_first_order` after `using KWave`.

The host side stays in Julia: the shim normalises the keyword arguments exactly where the
reference does, smooths p0 with `KWave.smooth(p0; restore_max=true)` in Float64 (as
initialize_p0_*! does), passes column-major arrays and `findall` indices (minus one) to the
library, and returns a `KWave.SimulationOutput` of Float64 arrays.  Fields and FFTs run in FP32
on the GPU whatever `data_cast` says.  libkwb.so is found at `ENV["KWB_LIBRARY"]` or next to the
Python host package (`k-wave-julia_b200/kwave_b200/libkwb.so`).
"""
module KWaveB200

using KWave

const libkwb = get(ENV, "KWB_LIBRARY", joinpath(@__DIR__, "..", "kwave_b200", "libkwb.so"))

const REC = Dict(:p => 0, :p_max => 1, :p_min => 2, :p_rms => 3, :p_final => 4, :ux => 5,
                 :uy => 6, :uz => 7, :u_max => 8, :u_rms => 9, :u_final => 10, :I_avg => 11,
                 :I_max => 12)
const SERIES = (:p, :ux, :uy, :uz)

struct KwbField
    data::Ptr{Float64}
    count::Int64
end
struct KwbSignal
    data::Ptr{Float64}
    n_rows::Int64
    n_cols::Int64
end
struct KwbSensorGroup
    index::Ptr{Int64}
    n_index::Int64
    dense::Int32
    cartesian::Int32
    record_mask::UInt32
    record_count::NTuple{13,UInt8}
    directivity_angle::Ptr{Float64}   # post-loop filters, applied on the device
    n_directivity_angle::Int64
    directivity_size::Float64
    has_frequency_response::Int32
    frequency_center::Float64
    frequency_bandwidth::Float64
end
struct KwbProblem
    ndim::Int32
    N::NTuple{3,Int64}
    d::NTuple{3,Float64}
    dt::Float64
    Nt::Int64
    pml_size::NTuple{3,Int64}
    pml_alpha::NTuple{3,Float64}
    c0::KwbField
    rho0::KwbField
    BonA::KwbField
    alpha_mode::Int32
    alpha_coeff::Float64
    alpha_power::Float64
    p0::KwbField
    p_index::Ptr{Int64}
    n_p_index::Int64
    p_mode::Int32
    p_signal::KwbSignal
    u_index::Ptr{Int64}
    n_u_index::Int64
    u_mode::Int32
    u_signal::NTuple{3,KwbSignal}
    tr::KwbSignal
    n_groups::Int32
    groups::Ptr{KwbSensorGroup}
    progress::Ptr{Cvoid}
    progress_user::Ptr{Cvoid}
    row_major::Int32  # 0: Julia arrays are column-major
    axisymmetric::Int32
    elastic::Int32
    cs::KwbField
    has_alpha_shear::Int32
    alpha_coeff_shear::Float64
    s_index::Ptr{Int64}
    n_s_index::Int64
    s_mode::Int32
    s_signal::NTuple{6,KwbSignal}
end
struct KwbGroupSizes
    rows::NTuple{13,Int64}
    cols::NTuple{13,Int64}
end
struct KwbGroupOutputs
    field::NTuple{13,Ptr{Float64}}
end
struct KwbOutputs
    groups::Ptr{KwbGroupOutputs}
    p_final_full::Ptr{Float64}
end

const CTX = Ref{Ptr{Cvoid}}(C_NULL)

function context()
    if CTX[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        rc = ccall((:kwb_context_create, libkwb), Cint, (Cint, Ref{Ptr{Cvoid}}), 0, h)
        rc == 0 || error(unsafe_string(ccall((:kwb_last_error, libkwb), Cstring, (Ptr{Cvoid},), C_NULL)))
        CTX[] = h[]
    end
    return CTX[]
end

check(rc) = rc == 0 ? rc :
    error(unsafe_string(ccall((:kwb_last_error, libkwb), Cstring, (Ptr{Cvoid},), context())))

# a scalar or array medium property (count 0 = nothing)
function field(x, keep)
    x === nothing && return KwbField(C_NULL, 0)
    v = x isa Real ? Float64[x] : vec(Float64.(x))   # column-major, like the reference
    push!(keep, v)
    return KwbField(pointer(v), length(v))
end

function signal(s, keep)
    s === nothing && return KwbSignal(C_NULL, 0, 0)
    m = s isa AbstractVector ? reshape(Float64.(s), :, 1) : Float64.(s)  # a Vector acts as n x 1
    push!(keep, m)
    return KwbSignal(pointer(m), size(m, 1), size(m, 2))
end

function indices(mask, keep)
    idx = Int64.(LinearIndices(mask)[findall(mask)]) .- 1
    push!(keep, idx)
    return idx
end

const _ALPHA = Dict(:no_absorption => 0, :no_dispersion => 1, :stokes => 2)

function _solve(kgrid, medium, source, sensor, pml_size, pml_alpha, smooth_p0, data_cast,
                progress_callback; axisymmetric::Bool=false, elastic::Bool=false)
    (kgrid.Nt[] == 0 || kgrid.dt[] == 0) &&
        error("Time array not set. Call make_time!(kgrid, sound_speed) before running.")
    data_cast == Float64 && @warn("KWaveB200 steps fields and FFTs in FP32 on the GPU; outputs stay " *
        "Float64 and agree with the reference's Float64 solve to about 1e-5 relative L2 " *
        "(data_cast = Float64 is not an FP64 GPU solve)") maxlog = 1
    KWave.validate_record_fields(sensor)
    dims = KWave.grid_size(kgrid)
    D = length(dims)
    ds = KWave.grid_spacing(kgrid)
    keep = Any[]
    psz = pml_size isa Tuple ? pml_size : ntuple(_ -> pml_size, D)
    pal = pml_alpha isa Tuple ? pml_alpha : ntuple(_ -> pml_alpha, D)
    pad3(t, v) = ntuple(i -> i <= D ? t[i] : v, 3)

    lossless = elastic || KWave.is_lossless(medium)
    if !lossless && !(medium.alpha_coeff isa Real)
        error("array alpha_coeff is not supported")          # T(absorb_tau) raises in the reference
    end
    # the axisymmetric and elastic solvers ignore time-reversal data
    tr = KWave.is_time_reversal(sensor) && !axisymmetric && !elastic
    p0 = KwbField(C_NULL, 0)
    if KWave.has_p0(source) && !tr
        q = Float64.(Array(source.p0))
        if !elastic && smooth_p0 && ((D == 1 && dims[1] > 4) || (D > 1 && all(>(1), dims)))
            q = KWave.smooth(q; restore_max=true)
        end
        p0 = field(q, keep)
    end
    has_p = !elastic && KWave.has_pressure_source(source)
    p_idx = has_p ? indices(source.p_mask, keep) : Int64[]
    u_idx = KWave.has_velocity_source(source) ? indices(source.u_mask, keep) : Int64[]
    psig = has_p ? signal(source.p, keep) : KwbSignal(C_NULL, 0, 0)
    usig = (signal(source.ux, keep), D > 1 ? signal(source.uy, keep) : KwbSignal(C_NULL, 0, 0),
            D > 2 ? signal(source.uz, keep) : KwbSignal(C_NULL, 0, 0))

    groups = KwbSensorGroup[]
    if sensor.mask !== nothing
        counts = zeros(UInt8, 13)
        mask = 0x00000000
        for f in sensor.record
            mask |= UInt32(1) << REC[f]
            counts[REC[f] + 1] += 1
        end
        if (:I_avg in sensor.record || :I_max in sensor.record) && data_cast == Float32 &&
           sensor.mask isa AbstractArray{Bool} && !elastic
            throw(MethodError(KWave._acoustic_intensity, (0.0f0,)))
        end
        if sensor.mask isa AbstractArray{Bool}
            idx = indices(sensor.mask, keep)
            dense = length(idx) == prod(dims)
            # post-loop filters (first_order_steps.jl:836-910), applied by libkwb before read-back
            ang_ptr, n_ang, dsize = Ptr{Float64}(C_NULL), Int64(0), 0.0
            if !elastic && sensor.directivity_angle !== nothing && sensor.directivity_size !== nothing
                ang = sensor.directivity_angle isa Real ? Float64[sensor.directivity_angle] :
                      collect(Float64, vec(sensor.directivity_angle))
                !(sensor.directivity_angle isa Real) && length(ang) < length(idx) &&
                    throw(BoundsError(sensor.directivity_angle, length(idx)))   # angle[j], first_order_steps.jl:853
                push!(keep, ang)
                ang_ptr, n_ang, dsize = pointer(ang), Int64(length(ang)), Float64(sensor.directivity_size)
            end
            has_fr = !elastic && sensor.frequency_response !== nothing
            fc, bw = has_fr ? Float64.(sensor.frequency_response) : (0.0, 0.0)
            push!(groups, KwbSensorGroup(dense ? C_NULL : pointer(idx), length(idx), Int32(dense), 0,
                                         mask, Tuple(counts), ang_ptr, n_ang, dsize, Int32(has_fr), fc, bw))
        else
            push!(groups, KwbSensorGroup(C_NULL, size(sensor.mask, 2), 0, 1, mask, Tuple(counts),
                                         C_NULL, 0, 0.0, 0, 0.0, 0.0))
        end
    end
    push!(keep, groups)
    trs = tr ? signal(sensor.time_reversal_boundary_data, keep) : KwbSignal(C_NULL, 0, 0)

    cb = C_NULL
    if progress_callback !== nothing
        fn = (t::Int64, Nt::Int64, p::Ptr{Float32}, ::Ptr{Cvoid}) ->
            (progress_callback(t, Nt, reshape(copy(unsafe_wrap(Array, p, prod(dims))), dims)); nothing)
        cfn = @cfunction($fn, Cvoid, (Int64, Int64, Ptr{Float32}, Ptr{Cvoid}))
        push!(keep, cfn)
        cb = Base.unsafe_convert(Ptr{Cvoid}, cfn)
    end

    nosig = KwbSignal(C_NULL, 0, 0)
    if elastic
        # ElasticMedium / ElasticSource (solver/elastic.jl:22-104); chi enters the 2D branch with a
        # scalar density only (elastic.jl:177-195, 282-295)
        used = D == 2 && medium.density isa Real
        y = medium.alpha_power
        absorb_p = used && y !== nothing && medium.alpha_coeff_compression !== nothing
        absorb_s = used && y !== nothing && medium.alpha_coeff_shear !== nothing
        c0f, rhof, bonaf = field(medium.sound_speed_compression, keep), field(medium.density, keep), KwbField(C_NULL, 0)
        amode, acoef, apow = absorb_p ? 1 : 0, absorb_p ? Float64(medium.alpha_coeff_compression) : 0.0,
                             y === nothing ? 0.0 : Float64(y)
        csf = field(medium.sound_speed_shear, keep)
        ashear = absorb_s ? Float64(medium.alpha_coeff_shear) : 0.0
        s_idx = KWave.has_stress_source(source) ? indices(source.s_mask, keep) : Int64[]
        comps = (source.sxx, source.syy, D > 2 ? source.szz : nothing, source.sxy,
                 D > 2 ? source.sxz : nothing, D > 2 ? source.syz : nothing)
        ssig = ntuple(k -> isempty(s_idx) ? nosig : signal(comps[k], keep), 6)
        smode = Int32(Int(source.s_mode))
    else
        c0f, rhof, bonaf = field(medium.sound_speed, keep), field(medium.density, keep), field(medium.BonA, keep)
        amode = lossless ? 0 : _ALPHA[medium.alpha_mode]
        acoef = lossless ? 0.0 : Float64(medium.alpha_coeff)
        apow = lossless ? 0.0 : Float64(medium.alpha_power)
        csf, absorb_s, ashear, s_idx, ssig, smode = KwbField(C_NULL, 0), false, 0.0, Int64[], ntuple(_ -> nosig, 6), Int32(0)
    end
    P = Ref(KwbProblem(Int32(D), pad3(dims, 1), pad3(ds, 1.0), kgrid.dt[], kgrid.Nt[],
                       pad3(psz, 0), pad3(Float64.(pal), 0.0),
                       c0f, rhof, bonaf, amode, acoef, apow, p0,
                       isempty(p_idx) ? C_NULL : pointer(p_idx), length(p_idx), has_p ? Int32(Int(source.p_mode)) : Int32(1), psig,
                       isempty(u_idx) ? C_NULL : pointer(u_idx), length(u_idx), Int32(Int(source.u_mode)), usig,
                       trs, length(groups), isempty(groups) ? C_NULL : pointer(groups), cb, C_NULL, Int32(0), Int32(axisymmetric),
                       Int32(elastic), csf, Int32(absorb_s), ashear,
                       isempty(s_idx) ? C_NULL : pointer(s_idx), length(s_idx), smode, ssig))
    ctx = context()
    GC.@preserve keep begin
        sizes = Vector{KwbGroupSizes}(undef, max(length(groups), 1))
        pf_len = Ref{Int64}(0)
        check(ccall((:kwb_query_outputs, libkwb), Cint,
                    (Ptr{Cvoid}, Ref{KwbProblem}, Ptr{KwbGroupSizes}, Ref{Int64}), ctx, P, sizes, pf_len))
        data = Dict{Symbol,AbstractArray}()
        outs = KwbGroupOutputs[]
        if !isempty(groups)
            ptrs = fill(Ptr{Float64}(C_NULL), 13)
            for f in unique(sensor.record)
                i = REC[f]
                a = zeros(Float64, sizes[1].rows[i + 1], sizes[1].cols[i + 1])
                data[f] = f in SERIES ? a : vec(a)
                ptrs[i + 1] = pointer(a)
            end
            push!(outs, KwbGroupOutputs(Tuple(ptrs)))
        end
        pfull = zeros(Float64, pf_len[])
        O = Ref(KwbOutputs(isempty(outs) ? C_NULL : pointer(outs), pf_len[] > 0 ? pointer(pfull) : C_NULL))
        GC.@preserve data outs pfull begin
            check(ccall((:kwb_solve, libkwb), Cint, (Ptr{Cvoid}, Ref{KwbProblem}, Ref{KwbOutputs}), ctx, P, O))
        end
    end
    if tr
        kgrid.Nt[] = size(sensor.time_reversal_boundary_data, 2)   # first_order.jl:430-431
        data[:p_final] = pfull
    end
    # the post-loop filters (apply_sensor_directivity!, apply_frequency_response!) ran in libkwb
    # on the device before read-back; the elastic solvers have none
    return KWave.SimulationOutput(data)
end

"""
    kspace_first_order(kgrid, medium, source, sensor; kwargs...) -> SimulationOutput

Same arguments and output as `KWave.kspace_first_order`; the time loop runs on the GPU.
`pml_inside`, `smooth_c0`, `smooth_rho0`, `plot_*`, `record_movie` and `show_progress` are
accepted and ignored, as in the reference solver body; `save_to_disk` is not supported.
"""
function kspace_first_order(kgrid::KWave.AbstractKWaveGrid, medium::KWave.KWaveMedium,
                            source::KWave.KWaveSource, sensor::KWave.KWaveSensor;
                            pml_inside::Bool=true, pml_size=20, pml_alpha=2.0, smooth_p0::Bool=true,
                            smooth_c0::Bool=false, smooth_rho0::Bool=false,
                            data_cast::Type{T}=Float64, save_to_disk=nothing, plot_sim::Bool=false,
                            plot_layout::Symbol=:default, plot_scale=:auto, record_movie=nothing,
                            progress_callback=nothing, show_progress::Bool=true) where {T<:AbstractFloat}
    save_to_disk === nothing || error("save_to_disk (HDF5 input files) is not supported by KWaveB200")
    return _solve(kgrid, medium, source, sensor, pml_size, pml_alpha, smooth_p0, T, progress_callback)
end

"""
    kspace_first_order_as(kgrid, medium, source, sensor; kwargs...) -> SimulationOutput

Same arguments and output as `KWave.kspace_first_order_as` (2D grid, x axial, y radial); the time
loop runs on the GPU.
"""
function kspace_first_order_as(kgrid::KWave.KWaveGrid2D, medium::KWave.KWaveMedium,
                               source::KWave.KWaveSource, sensor::KWave.KWaveSensor;
                               pml_inside::Bool=true, pml_size=20, pml_alpha=2.0,
                               smooth_p0::Bool=true, smooth_c0::Bool=false, smooth_rho0::Bool=false,
                               data_cast::Type{T}=Float64, plot_sim::Bool=false,
                               plot_layout::Symbol=:default, plot_scale=:auto,
                               record_movie=nothing, progress_callback=nothing) where {T<:AbstractFloat}
    return _solve(kgrid, medium, source, sensor, pml_size, pml_alpha, smooth_p0, T, progress_callback;
                  axisymmetric=true)
end

"""
    pstd_elastic_2d(kgrid, medium, source, sensor; kwargs...) -> SimulationOutput

Same arguments and output as `KWave.pstd_elastic_2d` (solver/elastic.jl:133-366); the time loop
runs on the GPU.  A scalar density with array wave speeds is rejected (the reference evaluates
`cp^2` as a matrix power there).
"""
function pstd_elastic_2d(kgrid::KWave.KWaveGrid2D, medium::KWave.ElasticMedium,
                         source::KWave.ElasticSource, sensor::KWave.KWaveSensor;
                         pml_size=20, pml_alpha=2.0, data_cast::Type{T}=Float64, plot_sim::Bool=false,
                         progress_callback=nothing) where {T<:AbstractFloat}
    return _solve(kgrid, medium, source, sensor, pml_size, pml_alpha, false, T, progress_callback;
                  elastic=true)
end

"""
    pstd_elastic_3d(kgrid, medium, source, sensor; kwargs...) -> SimulationOutput

Same arguments and output as `KWave.pstd_elastic_3d` (solver/elastic.jl:386-588).
"""
function pstd_elastic_3d(kgrid::KWave.KWaveGrid3D, medium::KWave.ElasticMedium,
                         source::KWave.ElasticSource, sensor::KWave.KWaveSensor;
                         pml_size=10, pml_alpha=2.0, data_cast::Type{T}=Float64, plot_sim::Bool=false,
                         progress_callback=nothing) where {T<:AbstractFloat}
    return _solve(kgrid, medium, source, sensor, pml_size, pml_alpha, false, T, progress_callback;
                  elastic=true)
end

end # module

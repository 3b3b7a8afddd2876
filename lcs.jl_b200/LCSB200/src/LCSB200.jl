"""
    LCSB200

B200 backend of LCS.jl.  The YAML `backend: {kind: b200}` selects it.  Every
function off the time step (init, statistics, HDF5 I/O, config) runs the
reference's own code on host arrays; `LCS.timestep` and `LCS.evolve!` call the
C ABI of liblcs_b200.so, which keeps the flow and particle state on the GPU.
"""
module LCSB200

using KernelAbstractions
using LCS
using PolySerde
using Topologies

include("abi.jl")

# A host-memory backend for the reference's own (non-hot-path) code.
struct B200Backend <: KernelAbstractions.GPU end
KernelAbstractions.zeros(::B200Backend, T, dims...) = zeros(T, dims...)
KernelAbstractions.allocate(::B200Backend, T, dims) = Array{T}(undef, dims)
KernelAbstractions.synchronize(::B200Backend) = nothing
Topologies.device!(::B200Backend; kwargs...) = nothing

PolySerde.@kind KernelAbstractions.Backend "b200" B200Backend
PolySerde.deserialize(::Type{B200Backend}, ::PolySerde.SerdeDict) = B200Backend()
PolySerde.serialize(::Type{B200Backend}, ::B200Backend, dicttype::PolySerde.SerdeDictType) = dicttype()

# foraxes on host arrays for the code that still runs in Julia (init, stats)
LCS.Parallel._foraxes(f, ::B200Backend, axes::Tuple{Vararg{AbstractUnitRange}}) =
    LCS.Parallel._foraxes(f, KernelAbstractions.CPU(), axes)

const HANDLES = IdDict{Any,Ptr{Cvoid}}()

const COLORINGS = Dict("NoColoring" => 0, "RedBlack" => 1, "RedBlackFast" => 2, "RedBlackBlock" => 3)

function lcs_config(config::LCS.Config)
    g = config.grid
    f = config.flow
    c = f.couple
    fk, power, energy, kmin, kmax, cs = 0, 0.0, 0.0, 0, 0, 0
    if f.forcing isa LCS.Flows.ConstantPowerLF
        fk, power = 1, f.forcing.power
    elseif f.forcing isa LCS.Flows.EnergyPreserveRCF
        fk, energy, kmin, kmax, cs = 2, f.forcing.energy, f.forcing.kmin, f.forcing.kmax, f.forcing.coarse_size
    end
    coloring = COLORINGS[string(nameof(typeof(c.coloring)))]
    block = c.coloring isa LCS.Parallel.RedBlackBlock ? c.coloring.size : 0
    parts = isnothing(config.particles) ? () : config.particles
    sp = ntuple(MAX_SPECIES) do s
        s <= length(parts) || return LcsSpecies(0, 0.0, 0.0, 0, 0)
        p = parts[s]
        LcsSpecies(LCS.Particles.nvalid_g(p.population), p.params.gravity, p.params.density_ratio,
                   p.drag isa LCS.Particles.NonlinearDrag ? 1 : 0, 0)
    end
    mode = config.mode isa LCS.FlowParticleMode ? 1 : 0
    LcsConfig(1, mode, Int32.(g.dims), g.halo_size, config.timestep.cfl, config.timestep.dtmax,
              f.params.U0_m_s, f.params.L0_m, f.params.NU_m2_s, c.time_blocking, c.overlap, coloring, block,
              c.omega, c.epsp, c.itrmin, c.itrmax, fk, kmin, kmax, cs, power, energy, length(parts), 0, sp, 0, 1)
end

# Upload the host state the reference's init! produced (once per buffer).
function handle(buf, state, config)
    get!(HANDLES, buf) do
        h = create(lcs_config(config))
        fl = buf.flow.fields
        un(A) = Array(LCS.unhalo(A, config.grid))
        upload_flow!(h, un(fl.Us[1]), un(fl.Us[2]), un(fl.Us[3]), un(fl.P))
        if !isnothing(buf.particles)
            for (s, pb) in enumerate(buf.particles)
                n = state.particles[s].nvalid
                pr = pb.props
                v(A) = Array(view(A, 1:n))
                upload_particles!(h, s - 1, v(pr.ids), v(pr.diams), v(pr.xss[1]), v(pr.xss[2]), v(pr.xss[3]),
                                  v(pr.uss[1]), v(pr.uss[2]), v(pr.uss[3]))
            end
        end
        set_state!(h, state.step, state.t)
        h
    end
end

# Copy the device state back into the reference's buffers (before stat/saverestart).
function download!(buf, state, config)
    h = HANDLES[buf]
    fl = buf.flow.fields
    dims = config.grid.dims
    U, V, W, P = (Array{Float64}(undef, dims...) for _ in 1:4)
    download_flow!(h, U, V, W, P)
    for (A, B) in zip((fl.Us..., fl.P), (U, V, W, P))
        LCS.unhalo(A, config.grid) .= B
    end
    if !isnothing(buf.particles)
        for (s, pb) in enumerate(buf.particles)
            n = state.particles[s].nvalid
            pr = pb.props
            ids = Vector{Int64}(undef, n)
            d, x, y, z, u, v, w = (Vector{Float64}(undef, n) for _ in 1:7)
            download_particles!(h, s - 1, ids, d, x, y, z, u, v, w)
            for (A, B) in zip((pr.ids, pr.diams, pr.xss..., pr.uss...), (ids, d, x, y, z, u, v, w))
                view(A, 1:n) .= B
            end
        end
    end
end

const B200Config = LCS.Config{<:Any,B200Backend}

# src/timestep.jl:14-18
LCS.timestep(::LCS.Mode, buf::LCS.Buffer, state::LCS.State, config::B200Config, topo::Topologies.Topology) =
    timestep(handle(buf, state, config))

# src/evolve.jl:63-146: one RK2 step on the device; the log mirrors the reference's NamedTuple
function LCS.evolve!(::LCS.Mode, buf::LCS.Buffer, state::LCS.State, config::B200Config, topo::Topologies.Topology;
                     kwargs...)
    lg = evolve!(handle(buf, state, config), state.dt)
    LCS.evolve!(state)
    (; flow=(; couple1=(; itr=Int(lg.couple1.itr), div=lg.couple1.div),
               couple2=(; itr=Int(lg.couple2.itr), div=lg.couple2.div),
               forcing=isnan(lg.p) ? LCS.EMPTY_LOG : isnan(lg.e10) ? (; p=lg.p) : (; p=lg.p, e10=lg.e10)))
end

# statistics and restart files read the reference's buffers: refresh them first
function LCS.stat(buf::LCS.Buffer, state::LCS.State, config::B200Config, topo::Topologies.Topology)
    download!(buf, state, config)
    invoke(LCS.stat, Tuple{LCS.Buffer,LCS.State,LCS.Config,Topologies.Topology}, buf, state, config, topo)
end

# src/LCSIO/save.jl:40-43: a restart step need not be a statistics step
function LCS.LCSIO.saverestart(buf::LCS.Buffer, state::LCS.State, config::B200Config, topo::Topologies.Topology)
    download!(buf, state, config)
    invoke(LCS.LCSIO.saverestart, Tuple{LCS.Buffer,LCS.State,LCS.Config,Topologies.Topology}, buf, state, config, topo)
end

end # module LCSB200

# ccall bindings of include/lcs_b200.h (the C ABI of liblcs_b200.so).
# LCS_B200_LIBRARY names the built library when LCSB200/ is copied beside
# LCSCUDA/ in an LCS.jl checkout (its [sources] paths assume that place).
const LIB = get(ENV, "LCS_B200_LIBRARY", joinpath(@__DIR__, "..", "..", "liblcs_b200.so"))
const MAX_SPECIES = 16

struct LcsSpecies
    nvalid::Int64
    gravity::Float64
    density_ratio::Float64
    drag::Int32
    _pad::Int32
end

struct LcsConfig
    abi_version::Int32
    mode::Int32
    dims::NTuple{3,Int32}
    halo_size::Int32
    cfl::Float64
    dtmax::Float64
    U0::Float64
    L0::Float64
    NU::Float64
    time_blocking::Int32
    overlap::Int32
    coloring::Int32
    coloring_block::Int32
    omega::Float64
    epsp::Float64
    itrmin::Int32
    itrmax::Int32
    forcing::Int32
    kmin::Int32
    kmax::Int32
    coarse_size::Int32
    power::Float64
    energy::Float64
    n_species::Int32
    precision::Int32
    species::NTuple{MAX_SPECIES,LcsSpecies}
    device::Int32
    use_graphs::Int32
end

struct LcsCoupleLog
    itr::Int32
    sweeps::Int32
    div::Float64
end

struct LcsLog
    couple1::LcsCoupleLog
    couple2::LcsCoupleLog
    p::Float64
    e10::Float64
    dt::Float64
    t::Float64
    step::Int64
end

lasterror(h) = unsafe_string(ccall((:lcs_last_error, LIB), Cstring, (Ptr{Cvoid},), h))
check(h, rc) = rc == 0 || throw(ArgumentError("lcs_b200: " * lasterror(h)))

function create(cfg::LcsConfig)
    r = Ref{Ptr{Cvoid}}(C_NULL)
    check(C_NULL, ccall((:lcs_create, LIB), Cint, (Ref{LcsConfig}, Ref{Ptr{Cvoid}}), cfg, r))
    r[]
end
destroy(h) = ccall((:lcs_destroy, LIB), Cvoid, (Ptr{Cvoid},), h)

upload_flow!(h, U, V, W, P) = check(h, ccall((:lcs_upload_flow, LIB), Cint,
    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h, U, V, W, P))
download_flow!(h, U, V, W, P) = check(h, ccall((:lcs_download_flow, LIB), Cint,
    (Ptr{Cvoid}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h, U, V, W, P))

function upload_particles!(h, s, ids, diam, x, y, z, u, v, w)
    n = length(x)
    check(h, ccall((:lcs_upload_particles, LIB), Cint,
        (Ptr{Cvoid}, Int32, Int64, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h, s, n, ids, diam, x, y, z, u, v, w))
end
function download_particles!(h, s, ids, diam, x, y, z, u, v, w)
    check(h, ccall((:lcs_download_particles, LIB), Cint,
        (Ptr{Cvoid}, Int32, Ptr{Int64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64}, Ptr{Float64},
         Ptr{Float64}, Ptr{Float64}, Ptr{Float64}), h, s, ids, diam, x, y, z, u, v, w))
end

function timestep(h)
    dt = Ref{Float64}()
    check(h, ccall((:lcs_timestep, LIB), Cint, (Ptr{Cvoid}, Ref{Float64}), h, dt))
    dt[]
end
function evolve!(h, dt::Float64)
    lg = Ref{LcsLog}()
    check(h, ccall((:lcs_evolve, LIB), Cint, (Ptr{Cvoid}, Float64, Ref{LcsLog}), h, dt, lg))
    lg[]
end
function step!(h, n::Integer)
    logs = Vector{LcsLog}(undef, n)
    check(h, ccall((:lcs_step, LIB), Cint, (Ptr{Cvoid}, Int32, Ptr{LcsLog}), h, n, logs))
    logs
end
set_state!(h, step, t) = check(h, ccall((:lcs_set_state, LIB), Cint, (Ptr{Cvoid}, Int64, Float64), h, step, t))

# ---- cell index and particle statistics (include/lcs_b200.h) -------------
const RDF_MAX_BINS = 1024
const SPECTRUM_MAX_SHELLS = 19
struct LcsParticleStatConfig
    grid_ratio::Int32
    bin_size::Int32
    search_cell_size::Int32
    max_wavenumber::Int32
    nsamples::Int32
    pad_::Int32
    contact_tolerance::Float64
    min_radius::Float64
end
struct LcsSummary
    mean::Float64
    max::Float64
    min::Float64
end
struct LcsParticleStats
    x::LcsSummary; y::LcsSummary; z::LcsSummary
    u::LcsSummary; v::LcsSummary; w::LcsSummary
    diam::LcsSummary
    taup::Float64
    St::Float64
    gr_contact::Float64
    npairs_contact::Int64
    nbins::Int32
    nshells::Int32
    edges::NTuple{RDF_MAX_BINS + 1,Float64}
    gr::NTuple{RDF_MAX_BINS,Float64}
    npairs::NTuple{RDF_MAX_BINS,Int64}
    wavenumbers::NTuple{SPECTRUM_MAX_SHELLS,Float64}
    Enp::NTuple{SPECTRUM_MAX_SHELLS,Float64}
end

makeindex!(h, s, stage, grid_ratio) =
    check(h, ccall((:lcs_particles_makeindex, LIB), Cint, (Ptr{Cvoid}, Int32, Int32, Int32), h, s, stage, grid_ratio))
# keep particles in cell order: makeindex! after every `interval`-th lcs_step step
set_particle_sort!(h, interval, grid_ratio) =
    check(h, ccall((:lcs_set_particle_sort, LIB), Cint, (Ptr{Cvoid}, Int32, Int32), h, interval, grid_ratio))
function particle_stat(h, s, pc::LcsParticleStatConfig, tau_eta::Float64)
    out = Ref{LcsParticleStats}()
    check(h, ccall((:lcs_particles_stat, LIB), Cint,
        (Ptr{Cvoid}, Int32, Ref{LcsParticleStatConfig}, Float64, Ref{LcsParticleStats}), h, s, pc, tau_eta, out))
    out[]
end
function particle_density(h, s, grid_ratio, n)
    rho = Vector{Float64}(undef, n)
    check(h, ccall((:lcs_particles_density, LIB), Cint, (Ptr{Cvoid}, Int32, Int32, Ptr{Float64}),
        h, s, grid_ratio, rho))
    rho
end

# ---- restart files (the reference's HDF5 layout, read and written by the library)
ioerror() = unsafe_string(ccall((:lcs_io_last_error, LIB), Cstring, ()))
checkio(rc) = rc == 0 || throw(ArgumentError("lcs_b200: " * ioerror()))
restart_save(h, path::AbstractString) = checkio(ccall((:lcs_restart_save, LIB), Cint, (Ptr{Cvoid}, Cstring), h, path))
restart_load!(h, path::AbstractString) = checkio(ccall((:lcs_restart_load, LIB), Cint, (Ptr{Cvoid}, Cstring), h, path))
restart_load_coarse!(h, path::AbstractString) =
    checkio(ccall((:lcs_restart_load_coarse, LIB), Cint, (Ptr{Cvoid}, Cstring), h, path))

# ---- the stat file (LCSIO.savestat of one step: state, stat and log)
struct LcsFlowStats
    u_mean::Float64; u_max::Float64; u_min::Float64
    v_mean::Float64; v_max::Float64; v_min::Float64
    w_mean::Float64; w_max::Float64; w_min::Float64
    k::Float64; epsilon::Float64; tau_eta::Float64; l_mu::Float64; l_eta::Float64; Re_lambda::Float64
    urms::Float64; k_eta::Float64; skewness::Float64; flatness::Float64; L::Float64; C_epsilon::Float64
end
function flow_stat(h)
    out = Ref{LcsFlowStats}()
    check(h, ccall((:lcs_flow_stat, LIB), Cint, (Ptr{Cvoid}, Ref{LcsFlowStats}), h, out))
    out[]
end
stat_save(path::AbstractString, step, t, dt, fs::LcsFlowStats, nvalid::Vector{Int64},
          ps::Vector{LcsParticleStats}, log::LcsLog) =
    checkio(ccall((:lcs_stat_save, LIB), Cint,
        (Cstring, Int64, Float64, Float64, Ref{LcsFlowStats}, Int32, Ptr{Int64}, Ptr{LcsParticleStats}, Ref{LcsLog}),
        path, step, t, dt, fs, length(ps), nvalid, ps, log))

"""
    GFB200

Julia-side binding of libgfb200.so: adds methods to `GeneralisedFilters.filter`
so that, for the model/algorithm combinations the B200 kernels implement, the
reference API `filter(rng, model, algo, ys)` runs on the GPU.  Everything else
keeps dispatching to the reference's CPU methods (this module adds methods; it
overrides none of the generic ones).

Not executed in this repository's CI (no Julia toolchain in the build image):
the same C entry points are exercised through Python ctypes in tests/.
"""
module GFB200

using GeneralisedFilters
using GeneralisedFilters: KalmanFilter, SRKalmanFilter, ParticleFilter, ESSResampler,
    Systematic, Stratified, Multinomial, LatentProposal, RBPF, HierarchicalSSM,
    ParticleDistribution, Particle, TypelessZero, AuxiliaryParticleFilter, MeanPredictive,
    ModePredictive, DrawPredictive, ConditionalSMC, NoRefreshment, AncestorSampling,
    BackwardSimulation
using SSMProblems
using Distributions: MvNormal
using LinearAlgebra
using Random

const libgfb200 = get(ENV, "GFB200_LIB", joinpath(@__DIR__, "..", "lib", "libgfb200.so"))

const GF_OK = Int32(0)
const GF_ERR_NOT_PD = Int32(1)
const GF_MEM_HOST = Int32(0)
const GF_PREC_F32, GF_PREC_F64 = Int32(0), Int32(1)
const GF_PROP_BOOTSTRAP = Int32(0)

# --- C structs (field order and types match include/gf_b200.h) ---------------
struct GfLgModel
    dx::Int32
    dy::Int32
    mu0::Ptr{Float64}
    Sigma0::Ptr{Float64}
    A::Ptr{Float64}
    b::Ptr{Float64}
    Q::Ptr{Float64}
    H::Ptr{Float64}
    c::Ptr{Float64}
    R::Ptr{Float64}
end

struct GfPfConfig
    n_particles::Int64
    resampler::Int32
    convention::Int32
    threshold::Float64
    precision::Int32
    proposal::Int32
    proposal_k::Float64
    seed::UInt64
    schedule::Ptr{Int8}
    lookahead::Int32   # GF_LOOKAHEAD_*
end

struct GfPfOut
    ll::Ptr{Float64}
    ll_steps::Ptr{Float64}
    ess_steps::Ptr{Float64}
    resampled::Ptr{Int8}
    ancestors::Ptr{Int32}
    means::Ptr{Float64}
    states::Ptr{Cvoid}
    log_weights::Ptr{Float64}
    clamps::Ptr{Int32}
    paths::Ptr{Cvoid}     # [T+1][dx][N] ancestry (AncestorCallback); C_NULL = off
    history::Ptr{Cvoid}   # [T+1][dx][N] states of every step (DenseAncestorCallback); C_NULL = off
    log_weight_history::Ptr{Float64}  # [T][N] normalised log-weights of every step; C_NULL = off
end

struct GfKfGradOut        # gf_kf_grad_out
    ll::Ptr{Float64}
    d_mu0::Ptr{Float64}
    d_Sigma0::Ptr{Float64}
    d_A::Ptr{Float64}
    d_b::Ptr{Float64}
    d_Q::Ptr{Float64}
    d_H::Ptr{Float64}
    d_c::Ptr{Float64}
    d_R::Ptr{Float64}
    status::Ptr{Int32}
end

struct GfCsmcConfig       # gf_csmc_config
    N::Int32
    threshold::Float64
    resampler::Int32
    refresh::Int32        # GF_CSMC_NONE / ANCESTOR / BACKWARD
    seed::UInt64
end

struct GfCsmcOut          # gf_csmc_out
    trajectories::Ptr{Float64}
    ll::Ptr{Float64}
    ref::Ptr{Float64}
    status::Ptr{Int32}
end

struct GfKfOut
    ll::Ptr{Float64}
    ll_steps::Ptr{Float64}
    means::Ptr{Float32}
    covs::Ptr{Float32}
    status::Ptr{Int32}
end

# --- context -------------------------------------------------------------------
const _ctx = Ref{Ptr{Cvoid}}(C_NULL)

function context()
    if _ctx[] == C_NULL
        h = Ref{Ptr{Cvoid}}(C_NULL)
        st = ccall((:gf_ctx_create, libgfb200), Int32, (Int32, Csize_t, Ref{Ptr{Cvoid}}), 0, 0, h)
        st == GF_OK || error("gf_ctx_create failed with status $st")
        _ctx[] = h[]
        atexit(() -> ccall((:gf_ctx_destroy, libgfb200), Int32, (Ptr{Cvoid},), _ctx[]))
    end
    return _ctx[]
end

function check(st::Int32)
    st == GF_OK && return nothing
    msg = unsafe_string(ccall((:gf_last_error, libgfb200), Cstring, (Ptr{Cvoid},), context()))
    st == GF_ERR_NOT_PD && throw(PosDefException(1))
    throw(ArgumentError("libgfb200 status $st: $msg"))
end

# --- model marshalling (Julia arrays are already column-major) ------------------
function lg_arrays(model)
    pr, dy, ob = SSMProblems.prior(model), SSMProblems.dyn(model), SSMProblems.obs(model)
    μ0, Σ0 = GeneralisedFilters.calc_initial(pr)
    A, b, Q = GeneralisedFilters.calc_params(dy, 1)
    H, c, R = GeneralisedFilters.calc_params(ob, 1)
    return map(x -> Matrix{Float64}(x isa AbstractVector ? reshape(x, :, 1) : Matrix(x)),
               (μ0, Σ0, A, b, Q, H, c, R))
end

function with_lg_model(f, model)
    arrs = lg_arrays(model)
    GC.@preserve arrs begin
        m = GfLgModel(Int32(size(arrs[3], 1)), Int32(size(arrs[6], 1)), map(pointer, arrs)...)
        return f(m)
    end
end

resampler_code(::Systematic) = Int32(0)
resampler_code(::Stratified) = Int32(1)
resampler_code(::Multinomial) = Int32(2)

# --- filter(model, KalmanFilter(), ys) -------------------------------------------
function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::GeneralisedFilters.LinearGaussianStateSpaceModel,
    algo::Union{KalmanFilter,SRKalmanFilter},
    observations::AbstractVector;
    callback=nothing,
    kwargs...,
)
    isnothing(callback) || throw(ArgumentError("GFB200 supports callback=nothing only"))
    T = length(observations)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    return with_lg_model(model) do m
        dx = Int(m.dx)
        ll = zeros(Float64, 1)
        means = zeros(Float32, dx * T)
        covs = zeros(Float32, dx * dx * T)
        status = zeros(Int32, 1)
        out = Ref(GfKfOut(pointer(ll), C_NULL, pointer(means), pointer(covs), pointer(status)))
        jit = algo.jitter
        GC.@preserve ll means covs status ys begin
            check(ccall((:gf_kf_batch, libgfb200), Int32,
                        (Ptr{Cvoid}, Int32, Ref{GfLgModel}, Int32, Ref{Int32}, Ptr{Float64},
                         Float64, Int32, Int32, Ref{GfKfOut}),
                        context(), algo isa KalmanFilter ? 0 : 1, m, 1, Int32(T), ys,
                        isnothing(jit) ? 0.0 : Float64(jit), isnothing(jit) ? 0 : 1,
                        GF_MEM_HOST, out))
        end
        μ = Float64.(means[(end - dx + 1):end])
        Σ = reshape(Float64.(covs[(end - dx * dx + 1):end]), dx, dx)
        return MvNormal(μ, Symmetric(Σ)), ll[1]
    end
end

# --- filter(rng, model, BF(N; threshold, resampler), ys) --------------------------
# AuxiliaryParticleFilter(BF(...), MeanPredictive() | ModePredictive() | DrawPredictive())
# takes the same call with the lookahead stage on (particles.jl:270-384); the draw comes
# from the library's own Philox stream, seeded from rng.
function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::GeneralisedFilters.LinearGaussianStateSpaceModel,
    algo::AuxiliaryParticleFilter{<:ParticleFilter{<:ESSResampler,LatentProposal}},
    observations::AbstractVector;
    kwargs...,
)
    pp = algo.weight_strategy.pp
    pp isa Union{MeanPredictive,ModePredictive,DrawPredictive} ||
        throw(ArgumentError("GFB200 builds the mean / mode / draw lookahead only"))
    return _bf(rng, model, algo.pf, observations, pp isa DrawPredictive ? Int32(2) : Int32(1);
               kwargs...)
end

function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::GeneralisedFilters.LinearGaussianStateSpaceModel,
    algo::ParticleFilter{<:ESSResampler,LatentProposal},
    observations::AbstractVector;
    kwargs...,
)
    return _bf(rng, model, algo, observations, Int32(0); kwargs...)
end

function _bf(rng, model, algo, observations, lookahead::Int32; callback=nothing, precision::Symbol=:f32,
             kwargs...)
    isnothing(callback) || throw(ArgumentError("GFB200 supports callback=nothing only"))
    N, T = algo.N, length(observations)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    cfg = Ref(GfPfConfig(N, resampler_code(algo.resampler.resampler), 0,
                         algo.resampler.threshold,
                         precision === :f64 ? GF_PREC_F64 : GF_PREC_F32, GF_PROP_BOOTSTRAP, 1.0,
                         rand(rng, UInt64), C_NULL, lookahead))
    return with_lg_model(model) do m
        dx = Int(m.dx)
        ET = precision === :f64 ? Float64 : Float32
        ll = zeros(Float64, 1)
        states = zeros(ET, N, dx)              # SoA [dx][N] == Matrix (N, dx)
        logw = zeros(Float64, N)
        out = Ref(GfPfOut(pointer(ll), C_NULL, C_NULL, C_NULL, C_NULL, C_NULL,
                          Ptr{Cvoid}(pointer(states)), pointer(logw), C_NULL, C_NULL, C_NULL, C_NULL))
        GC.@preserve ll states logw ys begin
            check(ccall((:gf_pf_run, libgfb200), Int32,
                        (Ptr{Cvoid}, Ref{GfLgModel}, Ref{GfPfConfig}, Int32, Ptr{Float64},
                         Ptr{Cvoid}, Ptr{Float64}, Int32, Ref{GfPfOut}),
                        context(), m, cfg, Int32(T), ys, C_NULL, C_NULL, GF_MEM_HOST, out))
        end
        particles = [Particle(Vector{ET}(states[i, :]), logw[i], 0) for i in 1:N]
        return ParticleDistribution(particles, zero(Float64)), ll[1]
    end
end

# --- kf_loglikelihood and its gradients (integrations/logdensity.jl:136-161) -------
"""
    kf_loglikelihood_grad(model, ys; jitter=nothing) -> (ll, grads)

kf_loglikelihood of a homogeneous linear-Gaussian model with the gradients its
ChainRules pullback returns for Δll = 1 (time-invariant parameters summed over t):
grads.μ0, .Σ0, .A, .b, .Q, .H, .c, .R.
"""
function kf_loglikelihood_grad(model, observations; jitter=nothing)
    T = length(observations)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    return with_lg_model(model) do m
        dx, dy = Int(m.dx), Int(m.dy)
        ll = zeros(1)
        g = (μ0=zeros(dx), Σ0=zeros(dx, dx), A=zeros(dx, dx), b=zeros(dx), Q=zeros(dx, dx),
             H=zeros(dy, dx), c=zeros(dy), R=zeros(dy, dy))
        status = zeros(Int32, 1)
        GC.@preserve ll g status ys begin
            out = Ref(GfKfGradOut(pointer(ll), pointer(g.μ0), pointer(g.Σ0), pointer(g.A), pointer(g.b),
                                  pointer(g.Q), pointer(g.H), pointer(g.c), pointer(g.R), pointer(status)))
            check(ccall((:gf_kf_loglikelihood_grad, libgfb200), Int32,
                        (Ptr{Cvoid}, Ref{GfLgModel}, Int32, Ref{Int32}, Ptr{Float64}, Float64, Int32, Int32,
                         Ref{GfKfGradOut}),
                        context(), m, 1, Int32(T), ys, isnothing(jitter) ? 0.0 : Float64(jitter),
                        isnothing(jitter) ? 0 : 1, GF_MEM_HOST, out))
        end
        return ll[1], g
    end
end

# --- conditional SMC (csmc.jl) -----------------------------------------------------
refresh_code(::NoRefreshment) = Int32(0)
refresh_code(::AncestorSampling) = Int32(1)
refresh_code(::BackwardSimulation) = Int32(2)

"""
    csmc_sample(rng, model, csmc::ConditionalSMC, observations, n; burnin=0, chains=1, init=nothing)

`n` kept sweeps of `chains` independent ConditionalSMC(BF(N; ...), refresh) chains
(bootstrap filter, linear-Gaussian model), each chain in one CUDA block.  Returns
(trajectories [dx, T+1, n, chains], lls [n, chains], last [dx, T+1, chains]); pass
`last` back as `init` to continue the chains.
"""
function csmc_sample(rng::AbstractRNG, model, csmc::ConditionalSMC, observations, n::Integer;
                     burnin::Integer=0, chains::Integer=1, init=nothing)
    pf = csmc.pf
    T = length(observations)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    cfg = Ref(GfCsmcConfig(Int32(pf.N), pf.resampler.threshold, resampler_code(pf.resampler.resampler),
                           refresh_code(csmc.refreshment), rand(rng, UInt64)))
    return with_lg_model(model) do m
        dx = Int(m.dx)
        trajs = zeros(dx, T + 1, n, chains)   # the C layout [chains][n][T+1][dx], column-major here
        lls = zeros(n, chains)
        ref = isnothing(init) ? zeros(dx, T + 1, chains) : Array{Float64}(init)
        status = zeros(Int32, chains)
        GC.@preserve trajs lls ref status ys begin
            out = Ref(GfCsmcOut(pointer(trajs), pointer(lls), pointer(ref), pointer(status)))
            check(ccall((:gf_csmc_run, libgfb200), Int32,
                        (Ptr{Cvoid}, Ref{GfLgModel}, Ref{GfCsmcConfig}, Int32, Ptr{Float64}, Int32, Int32,
                         Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Ref{GfCsmcOut}),
                        context(), m, cfg, Int32(T), ys, Int32(chains), Int32(burnin + n), Int32(burnin),
                        isnothing(init) ? 0 : 1, C_NULL, C_NULL, GF_MEM_HOST, out))
        end
        return trajs, lls, ref
    end
end

end # module

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
    BackwardSimulation, AbstractProposal
using GeneralisedFilters.GFTest: OptimalProposal, OverdispersedProposal, InnerDynamics
using SSMProblems
using Distributions: MvNormal
using LinearAlgebra
using Random

const libgfb200 = get(ENV, "GFB200_LIB", joinpath(@__DIR__, "..", "lib", "libgfb200.so"))

const GF_OK = Int32(0)
const GF_ERR_NOT_PD = Int32(1)
const GF_MEM_HOST = Int32(0)
const GF_PREC_F32, GF_PREC_F64 = Int32(0), Int32(1)
const GF_PROP_BOOTSTRAP, GF_PROP_OPTIMAL, GF_PROP_OVERDISPERSED = Int32(0), Int32(1), Int32(2)

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

struct GfRbModel          # gf_rb_model
    dxo::Int32
    dz::Int32
    dy::Int32
    mu_o::Ptr{Float64}
    Sigma_o::Ptr{Float64}
    A_o::Ptr{Float64}
    b_o::Ptr{Float64}
    Q_o::Ptr{Float64}
    mu_z::Ptr{Float64}
    Sigma_z::Ptr{Float64}
    A_z::Ptr{Float64}
    b_z::Ptr{Float64}
    C_z::Ptr{Float64}
    Q_z::Ptr{Float64}
    q_gamma::Float64
    q_index::Int32
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

# Time-varying models (any LinearGaussianLatentDynamics / ObservationProcess that
# is not the homogeneous type): calc_params(dyn, t), calc_params(obs, t) for
# t = 1..T stacked step-major (block t = step t, column-major) for the _tv entry
# points; f(m, param_steps).
is_homogeneous(model) = SSMProblems.dyn(model) isa GeneralisedFilters.HomogeneousLinearGaussianLatentDynamics &&
                        SSMProblems.obs(model) isa GeneralisedFilters.HomogeneousLinearGaussianObservationProcess

function with_lg_model_steps(f, model, T::Integer)
    is_homogeneous(model) && return with_lg_model(m -> f(m, Int32(1)), model)
    pr, dy, ob = SSMProblems.prior(model), SSMProblems.dyn(model), SSMProblems.obs(model)
    μ0, Σ0 = GeneralisedFilters.calc_initial(pr)
    col(x) = Float64.(vec(collect(x)))
    steps = [(GeneralisedFilters.calc_params(dy, t)..., GeneralisedFilters.calc_params(ob, t)...) for t in 1:T]
    stack(k) = reduce(vcat, [col(st[k]) for st in steps])
    arrs = (col(μ0), col(Matrix(Σ0)), stack(1), stack(2), stack(3), stack(4), stack(5), stack(6))
    dx, dyo = length(μ0), length(steps[1][5])
    GC.@preserve arrs begin
        m = GfLgModel(Int32(dx), Int32(dyo), map(pointer, arrs)...)
        return f(m, Int32(T))
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
    return with_lg_model_steps(model, T) do m, psteps
        dx = Int(m.dx)
        ll = zeros(Float64, 1)
        means = zeros(Float32, dx * T)
        covs = zeros(Float32, dx * dx * T)
        status = zeros(Int32, 1)
        out = Ref(GfKfOut(pointer(ll), C_NULL, pointer(means), pointer(covs), pointer(status)))
        jit = algo.jitter
        GC.@preserve ll means covs status ys begin
            # gf_kf_batch_tv with param_steps = 1 is gf_kf_batch
            check(ccall((:gf_kf_batch_tv, libgfb200), Int32,
                        (Ptr{Cvoid}, Int32, Ref{GfLgModel}, Int32, Ref{Int32}, Ref{Int32}, Ptr{Float64},
                         Float64, Int32, Int32, Ref{GfKfOut}),
                        context(), algo isa KalmanFilter ? 0 : 1, m, 1, Int32(T), psteps, ys,
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

# Guided filters (particles.jl:175-195) with the linear-Gaussian proposals the
# reference tests use: OptimalProposal (q = p(x_t | x_{t-1}, y_t), a Kalman update
# of N(A x + b, Q)) and OverdispersedProposal (N(A x + b, k Q)), GFTest/proposals.jl.
# The proposal's own dyn/obs must be the model's (as GFTest builds them).
function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::GeneralisedFilters.LinearGaussianStateSpaceModel,
    algo::ParticleFilter{<:ESSResampler,<:Union{OptimalProposal,OverdispersedProposal}},
    observations::AbstractVector;
    kwargs...,
)
    q = algo.proposal
    code = q isa OptimalProposal ? GF_PROP_OPTIMAL : GF_PROP_OVERDISPERSED
    k = q isa OverdispersedProposal ? Float64(q.k) : 1.0
    return _bf(rng, model, algo, observations, Int32(0); proposal=code, proposal_k=k, kwargs...)
end

# The reference's particles carry the model's element type: FP64 unless the
# model is Float32 (then the FP32-state / FP64-normaliser kernels run).
default_precision(model) = eltype(GeneralisedFilters.calc_params(SSMProblems.dyn(model), 1)[1]) === Float32 ?
                           :f32 : :f64

function _bf(rng, model, algo, observations, lookahead::Int32; callback=nothing,
             precision::Union{Symbol,Nothing}=nothing, proposal::Int32=GF_PROP_BOOTSTRAP,
             proposal_k::Float64=1.0, kwargs...)
    isnothing(callback) || throw(ArgumentError("GFB200 supports callback=nothing only"))
    precision = isnothing(precision) ? default_precision(model) : precision
    N, T = algo.N, length(observations)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    cfg = Ref(GfPfConfig(N, resampler_code(algo.resampler.resampler), 0,
                         algo.resampler.threshold,
                         precision === :f64 ? GF_PREC_F64 : GF_PREC_F32, proposal, proposal_k,
                         rand(rng, UInt64), C_NULL, lookahead))
    return with_lg_model_steps(model, T) do m, psteps
        dx = Int(m.dx)
        ET = precision === :f64 ? Float64 : Float32
        ll = zeros(Float64, 1)
        states = zeros(ET, N, dx)              # SoA [dx][N] == Matrix (N, dx)
        logw = zeros(Float64, N)
        out = Ref(GfPfOut(pointer(ll), C_NULL, C_NULL, C_NULL, C_NULL, C_NULL,
                          Ptr{Cvoid}(pointer(states)), pointer(logw), C_NULL, C_NULL, C_NULL, C_NULL))
        GC.@preserve ll states logw ys begin
            # gf_pf_run_tv with param_steps = 1 is gf_pf_run
            check(ccall((:gf_pf_run_tv, libgfb200), Int32,
                        (Ptr{Cvoid}, Ref{GfLgModel}, Int32, Ref{GfPfConfig}, Int32, Ptr{Float64},
                         Ptr{Cvoid}, Ptr{Float64}, Int32, Ref{GfPfOut}),
                        context(), m, psteps, cfg, Int32(T), ys, C_NULL, C_NULL, GF_MEM_HOST, out))
        end
        particles = [Particle(Vector{ET}(states[i, :]), logw[i], 0) for i in 1:N]
        return ParticleDistribution(particles, zero(Float64)), ll[1]
    end
end

# --- filter_batch(models, KalmanFilter() | SRKF(), yss) -----------------------------
"""
    filter_batch(models, algo::Union{KalmanFilter,SRKalmanFilter}, yss) -> Vector{(MvNormal, ll)}

B independent homogeneous linear-Gaussian models of uneven dx, dy and length,
filtered in one batched launch (gf_kf_batch); element f equals
`filter(models[f], algo, yss[f])`.
"""
function filter_batch(models::AbstractVector, algo::Union{KalmanFilter,SRKalmanFilter},
                      yss::AbstractVector)
    B = length(models)
    length(yss) == B || throw(ArgumentError("one observation sequence per model"))
    arrs = [lg_arrays(m) for m in models]
    Ts = Int32[length(y) for y in yss]
    ys = reduce(vcat, [reduce(vcat, [Float64.(collect(y)) for y in ysf]) for ysf in yss])
    dxs = [size(a[3], 1) for a in arrs]
    ll = zeros(Float64, B)
    means = zeros(Float32, sum(Int.(Ts) .* dxs))
    covs = zeros(Float32, sum(Int.(Ts) .* dxs .^ 2))
    status = zeros(Int32, B)
    jit = algo.jitter
    GC.@preserve arrs ll means covs status ys begin
        ms = [GfLgModel(Int32(size(a[3], 1)), Int32(size(a[6], 1)), map(pointer, a)...) for a in arrs]
        out = Ref(GfKfOut(pointer(ll), C_NULL, pointer(means), pointer(covs), pointer(status)))
        check(ccall((:gf_kf_batch, libgfb200), Int32,
                    (Ptr{Cvoid}, Int32, Ptr{GfLgModel}, Int32, Ptr{Int32}, Ptr{Float64},
                     Float64, Int32, Int32, Ref{GfKfOut}),
                    context(), algo isa KalmanFilter ? 0 : 1, ms, Int32(B), Ts, ys,
                    isnothing(jit) ? 0.0 : Float64(jit), isnothing(jit) ? 0 : 1, GF_MEM_HOST, out))
    end
    res = Vector{Any}(undef, B)
    mo, co = 0, 0
    for f in 1:B
        dx, T = dxs[f], Int(Ts[f])
        mo += T * dx
        co += T * dx * dx
        μ = Float64.(means[(mo - dx + 1):mo])
        Σ = reshape(Float64.(covs[(co - dx * dx + 1):co]), dx, dx)
        res[f] = (MvNormal(μ, Symmetric(Σ)), ll[f])
    end
    return res
end

# --- filter(rng, ::HierarchicalSSM, RBPF(BF(N; ...), KalmanFilter()), ys) ----------------
# rbpf.jl:8-84 on a conditionally linear-Gaussian HierarchicalSSM (models/hierarchical.jl):
# homogeneous linear-Gaussian outer prior and dynamics, inner prior N(mu_z, Sigma_z),
# inner dynamics GFTest.InnerDynamics (z' = A z + b + C x_prev + N(0, Q)) or any
# homogeneous linear-Gaussian dynamics (C = 0), linear-Gaussian observations of z.
# q_scale = (gamma, i) multiplies the inner Q by exp(gamma * x_t[i]) (the
# stochastic-volatility form of the trend-inflation example); (0, 1) = off.
function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::HierarchicalSSM,
    algo::RBPF{<:ParticleFilter{<:ESSResampler,LatentProposal},<:KalmanFilter},
    observations::AbstractVector;
    callback=nothing,
    q_scale::Tuple{Real,Integer}=(0.0, 1),
    kwargs...,
)
    return _rbpf(rng, model, algo, observations, Int32(0); callback, q_scale)
end

# AuxiliaryParticleFilter(RBPF(BF(N; ...), KalmanFilter()), pp) (rbpf.jl:86-124):
# x* is the mean / mode (MeanPredictive, ModePredictive) or a draw (DrawPredictive,
# from the library's lookahead Philox stream) of each particle's outer transition,
# and log eta the inner Kalman update's log-likelihood of y_t after predicting to x*.
function GeneralisedFilters.filter(
    rng::AbstractRNG,
    model::HierarchicalSSM,
    algo::AuxiliaryParticleFilter{<:RBPF{<:ParticleFilter{<:ESSResampler,LatentProposal},<:KalmanFilter}},
    observations::AbstractVector;
    callback=nothing,
    q_scale::Tuple{Real,Integer}=(0.0, 1),
    kwargs...,
)
    pp = algo.weight_strategy.pp
    pp isa Union{MeanPredictive,ModePredictive,DrawPredictive} ||
        throw(ArgumentError("GFB200 builds the mean / mode / draw lookahead only"))
    return _rbpf(rng, model, algo.pf, observations, pp isa DrawPredictive ? Int32(2) : Int32(1);
                 callback, q_scale)
end

function _rbpf(rng, model, algo, observations, lookahead::Int32; callback=nothing,
               q_scale::Tuple{Real,Integer}=(0.0, 1))
    isnothing(callback) || throw(ArgumentError("GFB200 supports callback=nothing only"))
    pf = algo.pf
    N, T = pf.N, length(observations)
    mat(x) = Matrix{Float64}(x isa AbstractVector ? reshape(x, :, 1) : Matrix(x))
    μo, Σo = GeneralisedFilters.calc_initial(model.outer_prior)
    μz, Σz = GeneralisedFilters.calc_initial(GeneralisedFilters.inner_prior(model))
    idyn = GeneralisedFilters.inner_dyn(model)
    odyn, obs = model.outer_dyn, SSMProblems.obs(model)
    # step t's parameters (calc_params(., t)); a model that is not of the
    # homogeneous types runs time-varying, one block per step (gf_rbpf_run_tv)
    function step_params(t)
        Ao, bo, Qo = GeneralisedFilters.calc_params(odyn, t)
        Az, bz, Cz, Qz = if idyn isa InnerDynamics
            idyn.A, idyn.b, idyn.C, idyn.Q
        else
            A_, b_, Q_ = GeneralisedFilters.calc_params(idyn, t)
            A_, b_, zeros(size(A_, 1), length(μo)), Q_
        end
        H, c, R = GeneralisedFilters.calc_params(obs, t)
        return map(mat, (Ao, bo, Qo, Az, bz, Cz, Qz, H, c, R))
    end
    homog = odyn isa GeneralisedFilters.HomogeneousLinearGaussianLatentDynamics &&
            (idyn isa InnerDynamics || idyn isa GeneralisedFilters.HomogeneousLinearGaussianLatentDynamics) &&
            obs isa GeneralisedFilters.HomogeneousLinearGaussianObservationProcess
    psteps = homog ? 1 : T
    blocks = [step_params(t) for t in 1:psteps]
    stk(k) = reduce(vcat, [vec(b[k]) for b in blocks])  # step-major, each column-major
    sp = ntuple(stk, 10)
    arrs = (mat(μo), mat(Σo), sp[1], sp[2], sp[3], mat(μz), mat(Σz), sp[4], sp[5], sp[6], sp[7], sp[8],
            sp[9], sp[10])
    dxo, dz, dy = size(blocks[1][1], 1), size(blocks[1][4], 1), size(blocks[1][8], 1)
    ys = reduce(vcat, [Float64.(collect(y)) for y in observations])
    cfg = Ref(GfPfConfig(N, resampler_code(pf.resampler.resampler), 0, pf.resampler.threshold,
                         GF_PREC_F32, GF_PROP_BOOTSTRAP, 1.0, rand(rng, UInt64), C_NULL, lookahead))
    width = dxo + dz + dz * (dz + 1) ÷ 2    # packed device state: x, mu, Sigma upper by rows
    ll = zeros(Float64, 1)
    states = zeros(Float32, N, width)
    logw = zeros(Float64, N)
    GC.@preserve arrs ll states logw ys begin
        p = map(pointer, arrs)
        m = Ref(GfRbModel(Int32(dxo), Int32(dz), Int32(dy), p[1:11]..., Float64(q_scale[1]),
                          Int32(q_scale[2] - 1), p[12:14]...))
        out = Ref(GfPfOut(pointer(ll), C_NULL, C_NULL, C_NULL, C_NULL, C_NULL,
                          Ptr{Cvoid}(pointer(states)), pointer(logw), C_NULL, C_NULL, C_NULL, C_NULL))
        check(ccall((:gf_rbpf_run_tv, libgfb200), Int32,
                    (Ptr{Cvoid}, Ref{GfRbModel}, Int32, Ref{GfPfConfig}, Int32, Ptr{Float64}, Ptr{Cvoid},
                     Ptr{Float64}, Int32, Ref{GfPfOut}, Ptr{Float64}),
                    context(), m, Int32(psteps), cfg, Int32(T), ys, C_NULL, C_NULL, GF_MEM_HOST, out,
                    C_NULL))
    end
    particles = map(1:N) do i
        x = Vector{Float64}(states[i, 1:dxo])
        μ = Vector{Float64}(states[i, (dxo + 1):(dxo + dz)])
        Σ = zeros(dz, dz)
        k = dxo + dz
        for r in 1:dz, q in r:dz
            k += 1
            Σ[r, q] = Σ[q, r] = states[i, k]
        end
        Particle(GeneralisedFilters.RBState(x, MvNormal(μ, Symmetric(Σ))), logw[i], 0)
    end
    return ParticleDistribution(particles, zero(Float64)), ll[1]
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
    # a model not of the homogeneous types runs with one parameter block per step
    return with_lg_model_steps(model, T) do m, psteps
        dx = Int(m.dx)
        trajs = zeros(dx, T + 1, n, chains)   # the C layout [chains][n][T+1][dx], column-major here
        lls = zeros(n, chains)
        ref = isnothing(init) ? zeros(dx, T + 1, chains) : Array{Float64}(init)
        status = zeros(Int32, chains)
        GC.@preserve trajs lls ref status ys begin
            out = Ref(GfCsmcOut(pointer(trajs), pointer(lls), pointer(ref), pointer(status)))
            check(ccall((:gf_csmc_run_tv, libgfb200), Int32,
                        (Ptr{Cvoid}, Ref{GfLgModel}, Int32, Ref{GfCsmcConfig}, Int32, Ptr{Float64}, Int32,
                         Int32, Int32, Int32, Ptr{Float64}, Ptr{Float64}, Int32, Ref{GfCsmcOut}),
                        context(), m, psteps, cfg, Int32(T), ys, Int32(chains), Int32(burnin + n),
                        Int32(burnin), isnothing(init) ? 0 : 1, C_NULL, C_NULL, GF_MEM_HOST, out))
        end
        return trajs, lls, ref
    end
end

end # module

"""gfb200 -- host-side mirror of GeneralisedFilters' filtering API over the
B200 library libgfb200.so (C ABI in include/gf_b200.h).

    from gfb200 import *
    model = create_homogeneous_linear_gaussian_model(mu0, Sigma0, A, b, Q, H, c, R)
    state, ll = filter(model, KalmanFilter(), ys)
    state, ll = filter(model, BF(2**20, threshold=0.5), ys, seed=1)
"""
from ._lib import (Context, GFError, PosDefException, default_context, load)  # noqa: F401
from .algorithms import (APF, BF, KF, KS, PF, RBPF, SRKF, AlternatingResampler,  # noqa: F401
                         AuxiliaryParticleFilter, BootstrapFilter, DrawPredictive, ESSResampler,
                         KalmanFilter, KalmanSmoother, LatentProposal, MeanPredictive, ModePredictive,
                         Multinomial, OptimalProposal, OverdispersedProposal, ParticleFilter,
                         RepresentativeStateLookAhead, SRKalmanFilter, Stratified, Systematic)
from .filtering import (AncestorCallback, DenseAncestorCallback, DenseParticleContainer,  # noqa: F401
                        ParticleTree, get_ancestry, kf_loglikelihood_grad, kf_loglikelihood_grad_batch,
                        InformationLikelihood, backward_information_batch, two_filter_smooth_all)
from .filtering import (MvNormal, ParticleDistribution, ancestors_to_offspring, filter,  # noqa: F401
                        filter_batch, offspring_to_ancestors, rng_normals, sample_ancestors,
                        smooth, smooth_batch)
from .models import (HierarchicalSSM, HomogeneousGaussianPrior,  # noqa: F401
                     HomogeneousLinearGaussianLatentDynamics,
                     HomogeneousLinearGaussianObservationProcess, InnerDynamics, NonHomogeneousInnerDynamics,
                     LatentDynamics, NonHomogeneousLinearGaussianLatentDynamics,
                     NonHomogeneousLinearGaussianObservationProcess, ObservationProcess,
                     StatePrior, StateSpaceModel, create_homogeneous_linear_gaussian_model,
                     create_nonhomogeneous_linear_gaussian_model)
from .serving import Server  # noqa: F401,E402
from .csmc import (AncestorSampling, BackwardSimulation, ConditionalSMC, CSMCModel,  # noqa: F401,E402
                   CSMCState, NoRefreshment)

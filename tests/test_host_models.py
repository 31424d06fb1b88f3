"""The model classes' host code on the CPU: fit / estimate of every model,
down to the arguments of the engine call, with the engine call itself (the
solvers' ``_run``, which needs a GPU) replaced by a recorder that returns the
start point as the result.  Checks what reaches the C-ABI: masked data,
options, starting points, b1 and sigma maps, prior rows and surface tables."""
import numpy as np
import pytest

from gacelle_b200 import GacelleError, _lib, askadam_solver, mcmc_solver, phantoms
from gacelle_b200 import gpuJointR1R2starMapping, gpuNEXI, gpuNEXIrice, gpuR2starMapping


@pytest.fixture
def engine(monkeypatch):
    calls = []

    def adam_run(self, gxm, y, w, theta0, b1, sig, gidx, d3, opts, nm, np_, prior=None, surface=None):
        calls.append(dict(kind="askadam", y=y, w=w, theta0=theta0, b1=b1, sigma=sig, gidx=gidx, dims=d3,
                          opts=opts, nm=nm, np=np_, prior=prior, surface=surface, model=gxm.s.kind))
        nv = y.shape[1]
        th = np.zeros((np_, nv), np.float32) if theta0 is None else np.asarray(theta0, np.float32)
        return {"final_theta": th, "min_theta": th, "final_residual": np.zeros((nm, nv), np.float32),
                "min_residual": np.zeros((nm, nv), np.float32), "final_resloss": np.zeros(nv, np.float32),
                "min_resloss": np.zeros(nv, np.float32), "loss_history": np.zeros(opts.iteration + 1),
                "final_loss": 1.0, "final_loss_fidelity": 1.0, "final_loss_reg": 0.0, "min_loss": 1.0,
                "min_loss_fidelity": 1.0, "min_loss_reg": 0.0, "final_niteration": opts.iteration,
                "min_niteration": opts.iteration, "stop_reason": 0}

    def mcmc_run(self, model, y, w, x0, b1, names, fitting, want_post, is_global=None, stats=()):
        calls.append(dict(kind="mcmc", y=y, w=w, x0=x0, b1=b1, names=names, fitting=fitting, stats=list(stats)))
        nvar, nv = len(names), y.shape[1]
        x = np.asarray(x0, np.float32).reshape(nvar, -1)[:, :nv]
        return {"mean": x, "std": np.zeros_like(x), "posterior": None, "W": int(fitting.get("Nwalker", 1)),
                "ns": 1, "rep": 1, "is_global": [0] * nvar, **{m: x for m in stats}}

    monkeypatch.setattr(askadam_solver.askadam, "_run", adam_run)
    monkeypatch.setattr(mcmc_solver.mcmc, "_run", mcmc_run)
    return calls


def test_r2s_fit_estimate_and_mcmc(engine, tmp_path):
    mask = phantoms.ellipsoid_mask((10, 8, 6), 1.0)
    data, _ = phantoms.r2s_phantom(mask, 3)
    m = gpuR2starMapping(phantoms.R2S_TE)
    out = m.fit(data, mask, {"iteration": 10, "start": "default", "lambda": [1e-3], "regmap": ["R2star"]})
    c = engine[-1]
    assert c["model"] == _lib.MODEL_R2S and c["y"].shape == (12, int(mask.sum())) and c["dims"] == mask.shape
    assert c["opts"].n_reg == 1 and c["opts"].reg_param[0] == 1 and c["opts"].reg_type == _lib.REG_TV
    np.testing.assert_array_equal(c["theta0"], np.tile([[1.0], [30.0]], (1, c["y"].shape[1])))
    assert out["final"]["R2star"].shape == mask.shape and out["final"]["R2star"][~mask].max() == 0
    # estimate: data scaled, two slabs with halos, M0 scaled back, saved
    f = {"iteration": 10, "start": "prior", "NSegmentUser": 2, "segmentOverlap": 1,
         "outputFilename": str(tmp_path / "o.mat")}
    n0 = len(engine)
    est = m.estimate(data, mask, f)
    assert len(engine) - n0 == 2 and est["final"]["loss"].shape == (2,)
    assert (tmp_path / "o.mat").exists() and est["mask"].shape == mask.shape
    # mcmc: noise kept as a parameter
    m2 = gpuR2starMapping(phantoms.R2S_TE)
    m2.fit(data, mask, {"solver": "mcmc", "iteration": 20, "algorithm": "ensemble", "start": "default"})
    assert engine[-1]["kind"] == "mcmc" and engine[-1]["names"] == ["M0", "R2star", "noise"]


def test_r1r2s_b1_and_true_flip_angle(engine):
    y, _ = phantoms.r1r2s_volume(120, 4)
    data = y.T.reshape(6, 5, 4, 24, order="F")
    mask = np.ones((6, 5, 4), bool)
    m = gpuJointR1R2starMapping(phantoms.R1R2S_TE, phantoms.R1R2S_TR, phantoms.R1R2S_FA)
    b1 = np.random.default_rng(5).uniform(0.8, 1.2, (6, 5, 4))
    m.fit(data, mask, {"iteration": 5}, {"b1": b1})
    a = engine[-1]["b1"]
    tfa = b1[..., None, None] * np.deg2rad(phantoms.R1R2S_FA)
    m.fit(data, mask, {"iteration": 5}, {"trueFlipAngle": tfa})
    np.testing.assert_allclose(engine[-1]["b1"], a, rtol=1e-6)
    np.testing.assert_allclose(a, b1.ravel(order="F"), rtol=1e-6)
    out = m.estimate(data, mask, {"iteration": 5, "start": "prior"}, {"trueFlipAngle": tfa})
    assert out["final"]["M0"].shape == (6, 5, 4) and engine[-1]["theta0"].shape == (3, 120)
    # mcmc receives the same b1, and estimate rescales M0 in every metric
    m2 = gpuJointR1R2starMapping(phantoms.R1R2S_TE, phantoms.R1R2S_TR, phantoms.R1R2S_FA)
    est = m2.estimate(data, mask, {"solver": "mcmc", "iteration": 20, "algorithm": "ensemble",
                                   "metric": ["mean", "std"]}, {"trueFlipAngle": tfa})
    c = engine[-1]
    assert c["kind"] == "mcmc" and c["names"] == ["M0", "R1", "R2star", "noise"]
    np.testing.assert_allclose(np.asarray(c["b1"]).ravel(), b1.ravel(order="F"), rtol=1e-6)
    assert est["mean"]["M0"].shape == (6, 5, 4)


def test_nexi_paths(engine, tmp_path):
    import test_surface
    b = np.tile([1.0, 2.5, 4.0], 2)
    d = np.repeat([20.0, 35.0], 3)
    m = gpuNEXI(b, d)
    rng = np.random.default_rng(6)
    shape = (5, 4, 3)
    data = rng.uniform(0.2, 0.8, shape + (6,)) * np.linspace(1, 0.5, 6)
    mask = np.ones(shape, bool)
    base = {"iteration": 5, "start": "default", "lossFunction": "mse"}
    m.fit(data, mask, dict(base))
    assert engine[-1]["opts"].n_reg == 0 and engine[-1]["np"] == 4
    # prior: mu / sigma images per regmap name, grid offset from outside the mask
    mask2 = mask.copy()
    mask2[0, 0, 0] = False
    mu = {"fa": np.full(shape, 0.5), "ra": np.full(shape, 0.1)}
    sd = {"fa": np.full(shape, 0.1), "ra": np.full(shape, 0.05)}
    m.fit(data, mask2, dict(base, regularisationType="prior", regmap=["fa", "ra"], **{"lambda": [1e-3, 2e-3]}),
          None, {"mu": mu, "sigma": sd})
    c = engine[-1]
    assert c["opts"].reg_type == _lib.REG_PRIOR and c["prior"][0].shape == (2, int(mask2.sum()))
    assert c["prior"][2] == pytest.approx(1e-3 / mask2.sum() * 5 + 2e-3 / mask2.sum() * 2)
    with pytest.raises(GacelleError):
        m.fit(data, mask, dict(base, regularisationType="prior", **{"lambda": [1e-3]}), None, {"mu": mu})
    # surface: geometry from FreeSurfer files, one call per hemisphere with NSegmentUser = 2
    nv = test_surface.write_subject(str(tmp_path), nx=6, ny=5)
    sdata = rng.uniform(0.2, 0.8, (1, nv, 2, 6))
    smask = np.ones((1, nv, 2), bool)
    ex = {"surf_dir": str(tmp_path), "hemisphere": ["lh", "rh"]}
    n0 = len(engine)
    m.estimate(sdata, smask, ex, dict(base, dataType="surface", **{"lambda": [1e-3]}))
    c = engine[-1]
    assert len(engine) - n0 == 1 and c["opts"].reg_type == _lib.REG_SURFACE_TV and c["dims"] == (1, nv, 2)
    assert c["surface"][0].shape[1] == 2 * nv and c["surface"][0].max() < 2 * nv
    n0 = len(engine)
    m.estimate(sdata, smask, ex, dict(base, dataType="surface", NSegmentUser=2, **{"lambda": [1e-3]}))
    assert len(engine) - n0 == 2 and engine[-1]["dims"] == (1, nv, 1)
    # the prior on surface data (geometry-agnostic, NEXI/gpuNEXI.m:382-415): no mesh needed
    smu = {"fa": np.full((1, nv, 2), 0.5)}
    ssd = {"fa": np.full((1, nv, 2), 0.1)}
    m.estimate(sdata, smask, {"mu": smu, "sigma": ssd},
               dict(base, dataType="surface", regularisationType="prior", regmap=["fa"], **{"lambda": [1e-3]}))
    c = engine[-1]
    assert c["opts"].reg_type == _lib.REG_PRIOR and c["surface"] is None and c["prior"][0].shape == (1, 2 * nv)


def test_nexi_rice_fit_keeps_spatial_tv(engine):
    m = gpuNEXIrice([1.0, 2.5, 4.0], [20.0, 20.0, 20.0])
    shape = (4, 3, 2)
    data = np.random.default_rng(7).uniform(0.3, 0.8, shape + (3,))
    mask = np.ones(shape, bool)
    m.fit(data, mask, {"iteration": 5, "start": "default", "regularisationType": "prior", "dataType": "surface",
                       "lambda": [1e-3]}, {"sigma": np.full(shape, 0.05)})
    c = engine[-1]
    assert c["model"] == _lib.MODEL_NEXI_RICE and c["opts"].reg_type == _lib.REG_TV
    np.testing.assert_allclose(c["sigma"], 0.05)

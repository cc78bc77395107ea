"""Generates the committed golden fixtures under tests/golden/.

Two sources:

1. The reference's own goldens (gprx `compare/goldens/*.json`, produced by
   sklearn 1.6.1, libgp and GPyTorch), read from a checkout of the reference
   and rewritten into one flat schema: kernel as flattened prefix nodes,
   log-θ, data, and the expected moments / NLML / NLML gradient.  The pinned
   Xoshiro256++ outputs of gprx `src/rng.rs` (test `sequence_is_pinned`) are
   read from that source file too.
2. Fresh sklearn fixed-θ cases at larger n (the same construction as the
   reference's `compare/generate.py`: `GaussianProcessRegressor(optimizer=None)`),
   which also pin the noise gradient through a WhiteKernel term.

Usage:  python tests/golden/make_fixtures.py REFERENCE_CHECKOUT
Nothing at test time reads the reference; only these committed JSON files.
"""

import json
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SUM, PRODUCT, RBF, RBF_ARD, CONSTANT, PERIODIC = 1, 2, 10, 11, 12, 13


def leaf_nodes(leaf, d):
    """Prefix nodes and log-θ for one golden leaf record."""
    kind = leaf["type"]
    if kind in ("sum", "product"):
        nodes, theta = [], []
        for child in leaf["leaves"]:
            n, t = leaf_nodes(child, d)
            nodes += n
            theta += t
        return [[SUM if kind == "sum" else PRODUCT, len(leaf["leaves"])]] + nodes, theta
    if kind == "rbf":
        return [[RBF, 0]], [math.log(leaf["lengthscale"])]
    if kind == "constant":
        return [[CONSTANT, 0]], [math.log(leaf["constant"])]
    if kind == "periodic":
        return [[PERIODIC, 0]], [math.log(leaf["lengthscale"]), math.log(leaf["period"])]
    raise KeyError(kind)


def exact_cases(gold_dir):
    out = []
    for name in ["rbf_n2", "rbf_n3"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        out.append(dict(
            name=name, source="gprx compare/goldens/%s.json (sklearn %s)" % (name, g["sklearn_version"]),
            nodes=[[RBF, 0]], theta=[math.log(g["lengthscale"])], noise_variance=g["noise_variance"],
            n=g["n_rows"], d=g["n_cols"], x=g["x"], y=g["y"], q=g["xs_n_rows"], xs=g["xs"],
            mean=g["mean"], latent_variance=g["latent_variance"],
            observation_variance=g["observation_variance"],
            nlml=-g["log_marginal_likelihood"], grad_kernel=[-g["grad_log_lengthscale"]], grad_noise=None))
    for name in ["rbf_sum_n2", "constant_rbf_product_n2", "constant_rbf_plus_rbf_n2", "periodic_n2"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        d = g["n_cols"]
        if g["kernel"] == "leaf":
            nodes, theta = leaf_nodes(g["leaves"][0], d)
        else:
            nodes, theta = leaf_nodes({"type": g["kernel"], "leaves": g["leaves"]}, d)
        assert np.allclose(theta, g["theta"]), name
        out.append(dict(
            name=name, source="gprx compare/goldens/%s.json (sklearn %s)" % (name, g["sklearn_version"]),
            nodes=nodes, theta=theta, noise_variance=g["noise_variance"],
            n=g["n_rows"], d=d, x=g["x"], y=g["y"], q=g["xs_n_rows"], xs=g["xs"],
            mean=g["mean"], latent_variance=g["latent_variance"],
            observation_variance=g["observation_variance"],
            nlml=-g["log_marginal_likelihood"],
            grad_kernel=[-v for v in g["grad_theta"]] if g.get("grad_theta") else None,
            grad_noise=None))
    return out


def sklearn_cases():
    """Fixed-θ sklearn cases with the noise as a WhiteKernel term so its
    gradient is pinned too (sklearn's `alpha` carries no gradient)."""
    import sklearn
    from sklearn.gaussian_process import GaussianProcessRegressor
    from sklearn.gaussian_process.kernels import RBF as SkRBF
    from sklearn.gaussian_process.kernels import ConstantKernel, ExpSineSquared, WhiteKernel

    rs = np.random.RandomState(20240611)
    specs = []
    # (name, n, d, sklearn kernel, nodes, theta, noise)
    specs.append(("sk_rbf_n48_d2", 48, 2, SkRBF(0.8), [[RBF, 0]], [math.log(0.8)], 0.05))
    ls = np.array([0.7, 1.3, 2.1])
    specs.append(("sk_const_rbfard_n64_d3", 64, 3, ConstantKernel(1.7) * SkRBF(ls),
                  [[PRODUCT, 2], [CONSTANT, 0], [RBF_ARD, 3]],
                  [math.log(1.7)] + list(np.log(ls)), 0.02))
    specs.append(("sk_rbf_plus_periodic_n56_d1", 56, 1, SkRBF(1.1) + ExpSineSquared(0.9, 1.6),
                  [[SUM, 2], [RBF, 0], [PERIODIC, 0]],
                  [math.log(1.1), math.log(0.9), math.log(1.6)], 0.1))
    specs.append(("sk_rbf_plus_periodic_n40_d3", 40, 3, SkRBF(1.4) + ExpSineSquared(2.5, 1.9),
                  [[SUM, 2], [RBF, 0], [PERIODIC, 0]],
                  [math.log(1.4), math.log(2.5), math.log(1.9)], 1.0))
    ls8 = np.exp(rs.uniform(math.log(0.3), math.log(3.0), size=8))
    specs.append(("sk_const_rbfard_n96_d8", 96, 8, ConstantKernel(2.0) * SkRBF(ls8),
                  [[PRODUCT, 2], [CONSTANT, 0], [RBF_ARD, 8]],
                  [math.log(2.0)] + list(np.log(ls8)), 0.0025))
    out = []
    for name, n, d, kern, nodes, theta, noise in specs:
        x = rs.uniform(0.0, 5.0, size=(n, d)) if d != 8 else rs.standard_normal(size=(n, d))
        y = np.sin(x.sum(axis=1)) + 0.3 * rs.standard_normal(n)
        q = 9
        xs = rs.uniform(0.0, 5.0, size=(q, d)) if d != 8 else rs.standard_normal(size=(q, d))
        gp_white = GaussianProcessRegressor(kern + WhiteKernel(noise, noise_level_bounds="fixed"),
                                            alpha=0.0, optimizer=None, normalize_y=False)
        gp_white.fit(x, y)
        full_kernel = kern + WhiteKernel(noise)
        gp_grad = GaussianProcessRegressor(full_kernel, alpha=0.0, optimizer=None, normalize_y=False)
        gp_grad.fit(x, y)
        lml, grad = gp_grad.log_marginal_likelihood(gp_grad.kernel_.theta, eval_gradient=True)
        gp = GaussianProcessRegressor(kern, alpha=noise, optimizer=None, normalize_y=False)
        gp.fit(x, y)
        mean, std = gp.predict(xs, return_std=True)
        lat = std ** 2
        assert np.allclose(gp_grad.kernel_.theta[:-1], theta)
        out.append(dict(
            name=name, source="sklearn %s GaussianProcessRegressor(optimizer=None)" % sklearn.__version__,
            nodes=nodes, theta=list(map(float, theta)), noise_variance=noise,
            n=n, d=d, x=list(x.T.reshape(-1)), y=list(y), q=q, xs=list(xs.T.reshape(-1)),
            mean=list(mean), latent_variance=list(lat), observation_variance=list(lat + noise),
            nlml=-float(lml), grad_kernel=[-float(v) for v in grad[:-1]], grad_noise=-float(grad[-1])))
    return out


def fit_cases(gold_dir):
    out = []
    for name in ["forrester_rbf", "sphere_rbf_ard"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        d = g["n_cols"]
        if g["kernel"] == "rbf":
            nodes = [[RBF, 0]]
        else:
            nodes = [[RBF_ARD, d]]
        out.append(dict(
            name=name, source="gprx compare/goldens/%s.json (sklearn %s, L-BFGS-B fit)" % (name, g["sklearn_version"]),
            nodes=nodes, theta_init=[math.log(v) for v in g["lengthscales_init"]],
            noise_variance_init=g["noise_variance_init"], normalize_y=g["normalize_y"],
            lengthscales=g["lengthscales"], noise_variance=g["noise_variance"],
            n=g["n_rows"], d=d, x=g["x"], y=g["y"], q=g["xs_n_rows"], xs=g["xs"],
            mean=g["mean"], latent_variance=g["latent_variance"],
            observation_variance=g["observation_variance"], lml=g["log_marginal_likelihood"]))
    return out


def online_cases(gold_dir):
    out = []
    for name in ["online_libgp_forrester", "online_libgp_sphere"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        d = g["n_cols"]
        nodes = [[RBF_ARD, d]] if g["ard"] else [[RBF, 0]]
        out.append(dict(
            name=name, source="gprx compare/goldens/%s.json (%s)" % (name, g["source"]),
            nodes=nodes, theta=[math.log(v) for v in g["lengthscales"]],
            noise_variance=g["noise_variance"], n=g["n_rows"], d=d, x=g["x"], y=g["y"],
            q=g["xs_n_rows"], xs=g["xs"], start_n=g["start_n"], steps=g["steps"]))
    return out


def sparse_cases(gold_dir):
    out = []
    for name in ["sgpr_forrester", "sgpr_sphere"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        d = g["n_cols"]
        for k in g["kernels"]:
            if k["name"] not in ("rbf", "rbf_ard"):
                continue  # Matérn and White leaves are outside this backend
            nodes = [[RBF, 0]] if k["name"] == "rbf" else [[RBF_ARD, d]]
            out.append(dict(
                name="%s_%s" % (name, k["name"]), source="gprx compare/goldens/%s.json (GPyTorch SGPR)" % name,
                nodes=nodes, theta=[math.log(v) for v in k["lengthscales"]],
                noise_variance=g["noise_variance"], n=g["n_rows"], d=d, x=g["x"], y=g["y"],
                m=g["m"], z=g["z"], q=g["xs_n_rows"], xs=g["xs"],
                nlml=k["neg_log_marginal_likelihood"], mean=k["mean"],
                latent_variance=k["latent_variance"], observation_variance=k["observation_variance"]))
    return out


def online_sparse_cases(gold_dir):
    out = []
    for name in ["online_sgpr_forrester", "online_sgpr_sphere"]:
        g = json.load(open(os.path.join(gold_dir, name + ".json")))
        d = g["n_cols"]
        for k in g["kernels"]:
            if k["name"] not in ("rbf", "rbf_ard"):
                continue
            nodes = [[RBF, 0]] if k["name"] == "rbf" else [[RBF_ARD, d]]
            out.append(dict(
                name="%s_%s" % (name, k["name"]), source="gprx compare/goldens/%s.json (GPyTorch reassembly)" % name,
                nodes=nodes, theta=[math.log(v) for v in k["lengthscales"]],
                noise_variance=g["noise_variance"], n=g["n_rows"], d=d, x=g["x"], y=g["y"],
                m=g["m"], z=g["z"], start_n=g["start_n"], start_m=g["start_m"],
                q=g["xs_n_rows"], xs=g["xs"], ops=g["ops"], steps=k["steps"]))
    return out


def rng_pins(ref):
    src = open(os.path.join(ref, "src", "rng.rs")).read()
    pins = {}
    for seed in ("0", "42"):
        m = re.search(r"const SEED_%s: \[u64; 4\] = \[(.*?)\];" % seed, src, re.S)
        vals = [int(v.strip().replace("_", ""), 16) for v in m.group(1).split(",") if v.strip()]
        pins[seed] = [str(v) for v in vals]
    return dict(source="gprx src/rng.rs sequence_is_pinned", seeds=pins)


def dump(name, obj):
    path = os.path.join(HERE, name)
    with open(path, "w") as fh:
        json.dump(obj, fh, indent=1)
        fh.write("\n")
    print("wrote", path)


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <gprx checkout>")
    ref = sys.argv[1]
    gold = os.path.join(ref, "compare", "goldens")
    dump("exact_goldens.json", exact_cases(gold))
    dump("sklearn_goldens.json", sklearn_cases())
    dump("fit_goldens.json", fit_cases(gold))
    dump("online_goldens.json", online_cases(gold))
    dump("sgpr_goldens.json", sparse_cases(gold))
    dump("online_sgpr_goldens.json", online_sparse_cases(gold))
    dump("rng_pins.json", rng_pins(ref))


if __name__ == "__main__":
    main()

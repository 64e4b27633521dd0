"""Drive the Dirac/KvN oracle through a notebook's preparation and Run() iterations."""
from oracle.dirac4d import DiracOracle


def prepare(cfg, alias_init=False):
    o = DiracOracle(cfg["params"], kvn=cfg["kvn"])
    Ws = o.W
    kind = cfg["init"]
    if kind == "landau":
        o.landau_ground(cfg["B"], 0.0, 0.0)
    else:
        ux, uy = cfg["u"]
        o.particle_up(ux, uy, 0.0, 0.0, 2.2, 2.2)
    if kind in ("up", "landau"):
        for W in Ws:
            o.theta_to_p(W)
        o.boundary_p(Ws)
    else:
        for W in Ws:
            o.theta_to_p(W)
        for W in Ws:
            o.x_to_lambda(W)
        if kind == "filtered":
            o.projector(Ws, 1)
        for W in Ws:
            o.lambda_to_x(W)
    for k in (0, 5, 10, 15):
        o.real(Ws[k])
    n = o.normalize(Ws)
    return o, n


def run(o, cfg, iterations, alias_w21=True, bound_p=7.0, observe=False):
    Ws = o.pointers(alias_w21)
    norms, obs = [], []
    for _ in range(iterations):
        n, ob = o.run_iteration(Ws, filter_particle=cfg["filter"], bound_p=bound_p,
                                observe=observe)
        norms.append(n)
        obs.append(ob)
    return norms, obs

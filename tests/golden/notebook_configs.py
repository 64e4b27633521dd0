"""The reference notebooks' frame settings, transcribed for the golden tests.

Each entry restates cell 4 ("class frame(...)") and the
``Set_Initial_Condition*`` cell a notebook runs, under
``instances/WignerDirac4D_64_64/`` and ``instances/WignerDiracKvN4D_64_64/``
of cabrer7/PyWignerCUDA2.  ``init`` names the preparation sequence:

* ``up``        ParticleUp -> _Fourier_Theta_To_P -> boundary_p -> Real -> Normalize
* ``filtered``  ParticleUp -> Theta_To_P -> X_To_Lambda -> projector(+1)
                -> Lambda_To_X -> Real -> Normalize
* ``unfiltered``  as ``filtered`` without the projector (SternGerlach quotes it out)
* ``landau``    WignerLandaoGround(B) -> _Fourier_Theta_To_P -> boundary_p -> Real -> Normalize
"""

_BASE = dict(gridDIM_p_y=64, gridDIM_y=64, gridDIM_p_x=64, gridDIM_x=64,
             theta_y_amplitude=28., lambda_y_amplitude=6., theta_x_amplitude=28.,
             lambda_x_amplitude=6., c=1., HBar=1., mass=1.,
             potential_0_String="0.", potential_1_String="0.", potential_2_String="0.",
             potential_3_String="0.", D_1_potential_0_String="0.",
             D_1_potential_1_String="0.", D_1_potential_2_String="0.")


def _cfg(**kw):
    d = dict(_BASE)
    d.update(kw)
    return d


def _amps(p, x):
    return dict(p_y_amplitude=p, p_x_amplitude=p, y_amplitude=x, x_amplitude=x)


def _D(v):
    return dict(D_theta_x=v, D_theta_y=v, D_lambda_x=v, D_lambda_y=v)


NOTEBOOKS = {
    "instances/WignerDirac4D_64_64/X.ipynb": dict(
        kvn=False, init="up", u=(0.5, 0.0), filter=False,
        params=_cfg(dt=0.01, potential_0_String="0.5*x", D_1_potential_0_String="0.5",
                    **_amps(2.5, 14.), **_D(0.0002))),
    "instances/WignerDirac4D_64_64/Y.ipynb": dict(
        kvn=False, init="up", u=(0.0, 0.5), filter=False,
        params=_cfg(dt=0.01, potential_0_String="0.5*y", **_amps(2.5, 14.), **_D(0.0002))),
    "instances/WignerDirac4D_64_64/Free.ipynb": dict(
        kvn=False, init="up", u=(0.5, 0.0), filter=False,
        params=_cfg(dt=0.005, **_amps(2.6, 15.), **_D(0.0001))),
    "instances/WignerDirac4D_64_64/X2.ipynb": dict(
        kvn=False, init="up", u=(0.5, 0.0), filter=False,
        params=_cfg(dt=0.01, potential_0_String="0.04*pow(x-5.,2)",
                    D_1_potential_0_String="0.08*(x-5)", **_amps(2.9, 15.), **_D(0.0001))),
    "instances/WignerDirac4D_64_64/FreeFiltered.ipynb": dict(
        kvn=False, init="filtered", u=(0.5, 0.0), filter=False,
        params=_cfg(dt=0.01, **_amps(2.5, 14.), **_D(0.0002))),
    "instances/WignerDirac4D_64_64/X_Filtered.ipynb": dict(
        kvn=False, init="filtered", u=(0.5, 0.0), filter=True,
        params=_cfg(dt=0.01, potential_0_String="0.5*x", D_1_potential_0_String="0.5",
                    **_amps(2.5, 14.), **_D(0.0002))),
    "instances/WignerDirac4D_64_64/Landao.ipynb": dict(
        kvn=False, init="landau", B=0.26, filter=False,
        params=_cfg(dt=0.01, potential_1_String="-y*0.26/2.", potential_2_String="x*0.26/2.",
                    D_1_potential_2_String="0.26*0.5", **_amps(2.6, 17.), **_D(0.00001))),
    "instances/WignerDirac4D_64_64/Landao_X.ipynb": dict(
        kvn=False, init="landau", B=0.26, filter=False,
        params=_cfg(dt=0.01, potential_1_String="-y*0.26/2.",
                    potential_2_String="x*0.26/2. + 0.05*pow(x,2)",
                    D_1_potential_2_String="0.26*0.5 + 0.1*x", **_amps(2.6, 17.), **_D(0.00001))),
    "instances/WignerDirac4D_64_64/SternGerlach.ipynb": dict(
        kvn=False, init="unfiltered", u=(0.0, 0.0), filter=False,
        params=_cfg(dt=0.01, potential_3_String="y*(x+16)/50.", **_amps(2.5, 16.), **_D(0.0001))),
    "instances/WignerDiracKvN4D_64_64/Free_Vx.ipynb": dict(
        kvn=True, init="filtered", u=(0.5, 0.0), filter=True,
        params=_cfg(dt=0.01, **_amps(2.5, 14.), **_D(0.0001))),
    "instances/WignerDiracKvN4D_64_64/Free_Vy.ipynb": dict(
        kvn=True, init="filtered", u=(0.0, 0.5), filter=True,
        params=_cfg(dt=0.01, **_amps(2.5, 14.), **_D(0.0001))),
}

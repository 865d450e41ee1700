"""The reference's AD-OO oil-water model with its cell equations assembled on
the GPU: `use_device_cell_equations(model)` gives a
TwoPhaseOilWaterModel (pymrst/modules/ad_blackoil/models/
two_phase_oil_water_model.py) a `get_equations` that follows
equations_oil_water (pymrst/modules/ad_blackoil/utils/
equations_oil_water.py:17-72) with the water and oil cell equations - the
accumulation terms and the divergence of the upwinded surface-volume fluxes,
with their Jacobians in pressure and water saturation - formed by the
device oil-water kernels (`csrc/ow.cu`, a well-free model on the same grid,
fluid, transmissibilities and gravity).  Boundary conditions, sources and
the facility (well) equations are then added by the model's own methods,
and the problem is set up by the model, so the reference's AD-OO
NonLinearSolver, linear solvers and facility model work unchanged.

The AD-OO cell equations are the legacy model's (the same accumulation, the
same phase-upwinded fluxes), which the device kernels reproduce.  Requires a
vertical gravity vector and the simple AD fluid (init_simple_adi_fluid).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .ow_model import GpuOilWaterModel, OWState


_DEVICE = {}


def _device_model(model):
    """The well-free device model of the grid, rock, fluid, gravity and
    transmissibilities (cached by identity; the reference's drivers work on
    shallow copies of the model that share them)."""
    g = model.G
    gvec = np.asarray(model.get_gravity_vector(), dtype=float).ravel()
    if np.any(gvec[:-1] != 0.0):
        raise ValueError("device cell equations need a vertical gravity vector")
    ops = model.operators
    T = np.asarray(ops.T, dtype=float).ravel()
    key = (id(g), id(model.rock), id(model.fluid), tuple(gvec), hash(T.tobytes()))
    dev = _DEVICE.get(key)
    if dev is not None:
        return dev
    dev = GpuOilWaterModel(g, model.rock, model.fluid, [], gravity=float(gvec[-1]) if gvec.size else 0.0, T=T,
                           cpr_options=dict(rtol=1e-12))
    gdz = getattr(ops, "gdz", None)
    if gdz is not None and np.size(gdz) == dev.gdz.size:
        scale = max(np.abs(np.asarray(gdz, dtype=float)).max(), 1e-300)
        if np.abs(np.asarray(gdz, dtype=float).ravel() - dev.gdz).max() > 1e-12 * scale:
            raise ValueError("device cell equations: the model's gravity gradient is not g (z[N1] - z[N0])")
    if len(_DEVICE) >= 8:
        _DEVICE.pop(next(iter(_DEVICE)))
    _DEVICE[key] = dev
    return dev


def _cell_equations(model, p_now, sw_now, p_old, sw_old, dt, p_ad):
    """Water and oil cell equations (values and Jacobian blocks in pressure
    and water saturation) from the device, as AD values of the model's type
    with zero blocks for the facility unknowns."""
    import torch
    dev = _device_model(model)
    nc = dev.nc
    st = OWState(pressure=p_now, sW=sw_now, qWs=np.zeros(0), qOs=np.zeros(0), bhp=np.zeros(0))
    st0 = OWState(pressure=p_old, sW=sw_old, qWs=np.zeros(0), qOs=np.zeros(0), bhp=np.zeros(0))
    x, x0 = dev.to_device(st), dev.to_device(st0)
    cdp = torch.zeros(1, dtype=torch.float64, device="cuda")
    res, jac, well = dev.assemble_device(x, x0, float(dt), cdp, True)
    r = dev.export_residual(res.cpu().numpy())
    J = sp.csr_array(dev.export_jacobian(jac.cpu().numpy(), well.cpu().numpy()))
    ADI = type(p_ad)
    widths = [blk.shape[1] for blk in p_ad.jac]
    out = []
    for e in range(2):
        rows = slice(e * nc, (e + 1) * nc)
        blocks = [J[rows, 0:nc], J[rows, nc:2 * nc]]
        blocks += [sp.csr_array((nc, w)) for w in widths[2:]]
        out.append(ADI(r[rows], blocks))
    return out


def _get_equations(self, state0, state, dt, driving_forces, **options):
    from pymrst.modules.ad_core.ad_oo.physical_model import copy_state
    state = copy_state(state)
    state0 = copy_state(state0)
    num = lambda v: np.asarray(getattr(v, "val", v), dtype=float)
    p_now, p_old = num(state["pressure"]).ravel().copy(), num(state0["pressure"]).ravel().copy()
    sw_now = np.atleast_2d(num(state["s"]))[:, 0].copy()
    sw_old = np.atleast_2d(num(state0["s"]))[:, 0].copy()
    p, s_w, well_sol = self.get_props(state, "pressure", "water", "wellsol")
    p0, s_w0, well_sol0 = self.get_props(state0, "pressure", "water", "wellSol")
    well_vars, well_var_names, well_map = self.FacilityModel.get_all_primary_variables(well_sol)
    reverse, res_only = bool(options.get("reverseMode", False)), bool(options.get("resOnly", False))
    if res_only or reverse:
        raise NotImplementedError("device cell equations: residual-only and reverse modes are the reference's")
    p, s_w, *well_vars = self.AutoDiffBackend.init_variables_ad(p, s_w, *well_vars)
    primary = ["pressure", "sW"] + list(well_var_names)
    sat, sat0 = [s_w, 1 - s_w], [s_w0, 1 - s_w0]
    state = self.set_props(state, ["s", "pressure"], [sat, p])
    state0 = self.set_props(state0, ["s", "pressure"], [sat0, p0])
    state = self.init_state_function_containers(state)
    pressures, mob, rho = self.get_props(state, "PhasePressures", "Mobility", "Density")
    if self.outputFluxes or self.extraStateOutput:
        # output fields only: the host state functions, as the reference stores them
        b = self.get_props(state, "ShrinkageFactors")
        (v_w, v_o), (upcw, upco) = self.get_props(state, "PhaseFlux", "PhaseUpwindFlag")
        if self.outputFluxes:
            state = self.store_fluxes(state, v_w, v_o, None)
        if self.extraStateOutput:
            state = self.storebfactors(state, b[0], b[1], None)
            state = self.store_mobilities(state, *mob, None)
            state = self.store_upstream_indices(state, upcw, upco, None)
    water, oil = _cell_equations(self, p_now, sw_now, p_old, sw_old, dt, p)
    eqs, names, types_ = [water, oil], ["water", "oil"], ["cell", "cell"]
    eqs, state, _ = self.add_boundary_conditions_and_sources(eqs, names, types_, state, pressures, sat, mob, rho,
                                                             [], [], driving_forces)
    if self.AquiferModel is not None:
        raise NotImplementedError("device cell equations: aquifers are not supported")
    opt = {"iteration": options.get("iteration", -1), "reverseMode": False, "resOnly": False}
    eqs, names, types_, state["wellSol"], _ = self.insert_well_equations(
        eqs, names, types_, well_sol0, well_sol, well_vars, well_map, p, mob, rho, [], [], dt, opt)
    problem = self.setup_linearized_problem(eqs, types_, names, primary, state, dt)
    return problem, state


def use_device_cell_equations(model):
    """The model (the reference's AD-OO TwoPhaseOilWaterModel) with its
    get_equations assembling the cell equations on the GPU; returns it.  The
    model's class becomes a subclass with that method, so that the copies
    the reference's drivers make of the model keep it."""
    cls = type(model)
    if not getattr(cls, "_pmb_device_cells_class", False):
        cls = type("Gpu" + cls.__name__, (cls,), {"get_equations": _get_equations, "getEquations": _get_equations,
                                                  "_pmb_device_cells_class": True})
        model.__class__ = cls
    return model

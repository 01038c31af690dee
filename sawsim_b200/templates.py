"""Template cases from the reference's configuration fields, without Gmsh (host setup).

The reference builds a template's model from a configuration
(``src/sawsim/models.py:27-140`` for the Q9 templates,
``src/sawsim/hex_models.py:57-107`` for the Hex27 slabs): the mesh of the
template, the materials in the order substrate, electrode, backing layers,
coatings, the PML region below the last layer (2 pitches, the last backing's
material), the Bloch sets, and the loss settings.  ``case_for`` does the same
for the templates this package rebuilds without Gmsh -- ``sp_stack`` (any
stack), ``sp_double_layer`` and ``sp_quad_layer`` (their default geometry),
``sp_2p5d_{single,double,triple,quad}_layer`` -- and ``engine_for`` builds the
GPU engine of the result, Rayleigh damping included.

``materials`` are the resolved tensors in the reference's order (the substrate
already rotated by its Euler angles, as ``material_runtime.resolve_materials``
returns them); plane strain (``mode_extension`` 0) projects them onto the mesh
plane here, xz for the TC-SAW substrate ``linbo3_tc`` (models.py:64-66).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import cases, cells
from . import materials as mt

Q9_TEMPLATES = ('sp_stack', 'sp_double_layer', 'sp_quad_layer')
HEX_TEMPLATES = tuple(f'sp_2p5d_{k}_layer' for k in ('single', 'double', 'triple', 'quad'))
# the one geometry of each fixed structured template that cells rebuilds
_FIXED = {'sp_double_layer': dict(pitch_um=1.085, electrode_um=0.17, substrate_um=0.6, metal_ratio=0.5,
                                  mesh_um=0.5, layers=[8.33]),
          'sp_quad_layer': dict(pitch_um=1.085, electrode_um=0.17, substrate_um=0.6, metal_ratio=0.5,
                                mesh_um=0.5, layers=[0.5, 1.0, 7.83])}


@dataclass
class Loss:
    """Loss settings of a configuration (models.py:67-70, solver.py:109-115)."""

    beta_dk: float = 0.0          # Rayleigh stiffness damping of the piezo layer
    eta_eps: float = 0.0          # dielectric loss of the piezo layer, eps (1 - i eta)


def _thickness(layer):
    return float(layer['thickness_um'] if isinstance(layer, dict) else layer.thickness_um)


def _freqs(config):
    return np.linspace(config['start_ghz'] * 1e9, config['stop_ghz'] * 1e9, int(config['points']))


def case_for(config, materials: list):
    """``(case, loss)`` of a configuration (a dict of the reference's configuration
    fields, or its ``SimulationConfig``): a ``cases.Case`` (Q9) or ``cases.HexCase``."""
    if not isinstance(config, dict):
        config = config.model_dump()
    model_id = config['model_id']
    loss = Loss(float(config.get('beta_dk') or 0.0), float(config.get('eta_eps') or 0.0))
    layers = [_thickness(x) for x in config.get('layers', [])]
    coatings = [_thickness(x) for x in config.get('coatings', [])]
    mats = list(materials)
    if len(mats) != 2 + len(layers) + len(coatings):
        raise ValueError(f'{model_id}: {2 + len(layers) + len(coatings)} materials expected (substrate, electrode, '
                         f'{len(layers)} layers, {len(coatings)} coatings), {len(mats)} given')
    if loss.eta_eps:
        m = mats[0]
        mats[0] = mt.Material(m.rho, m.C, m.e, m.eps * (1 - 1j * loss.eta_eps))
    if model_id in HEX_TEMPLATES:
        kind = model_id[len('sp_2p5d_'):-len('_layer')]
        cell = cells.sp_2p5d_template_cell(kind, config['pitch_um'], config['electrode_um'], config['substrate_um'],
                                           layers, config['metal_ratio'], config['mesh_um'], config['aperture_um'])
        idx = np.array([cell.tag_map[int(t)] for t in cell.hex_tag], dtype=np.int64)
        pos_m = cell.POS * 1e-6
        bottom = float(pos_m[:, 2].min())
        pml = [cases.PML(tag=cell.pml_tag, kind='z', za=cell.pml_top_um * 1e-6, zp=bottom)]
        bc = cases.bc_periodic_3d(cell.sets, pos_m, pos_m.shape[0])
        return cases.HexCase(model_id, cell, pos_m, cell.HEXAS27, mats, idx, pml, bc, _freqs(config),
                             dict(config=config)), loss
    if model_id not in Q9_TEMPLATES:
        raise ValueError(f'{model_id}: no Gmsh-free rebuild (Q9: {Q9_TEMPLATES}; Hex27: {HEX_TEMPLATES})')
    if model_id == 'sp_stack':
        cell = cells.sp_stack_cell(config['pitch_um'], config['metal_ratio'], config['electrode_um'],
                                   config['substrate_um'], layers, coatings, config['mesh_um'])
    else:
        fixed = _FIXED[model_id]
        got = dict(pitch_um=config['pitch_um'], electrode_um=config['electrode_um'],
                   substrate_um=config['substrate_um'], metal_ratio=config['metal_ratio'], mesh_um=config['mesh_um'],
                   layers=layers)
        if any(not np.isclose(got[k], fixed[k]).all() for k in fixed):
            raise ValueError(f'{model_id} is rebuilt at its default geometry only; use sp_stack for other stacks')
        cell = cells.sp_double_layer_cell() if model_id == 'sp_double_layer' else cells.sp_quad_layer_cell()
    me = int(config.get('mode_extension', 1))
    if not me:
        project = (mt.project_xz_plane_strain if config.get('substrate_material') == 'linbo3_tc'
                   else mt.project_xy_plane_strain)
        mats = [project(m) for m in mats]
    mesh = cases.mesh_from_msh(cell.msh())
    idx = np.array([cell.tag_map[int(t)] for t in mesh.elem_tag], dtype=np.int64)
    bottom = float(mesh.pos_m[:, 1].min())
    pml = [cases.PML(tag=cell.pml_tag, kind='y', yp=bottom, ya=bottom + 2 * config['pitch_um'] * 1e-6)]
    bc = cases.bc_periodic(mesh, cell.LINES3, 3 if me else 2)
    return cases.Case(model_id, cell, mesh, mats, idx, pml, bc, _freqs(config), me, dict(config=config)), loss


def damping_materials(materials: list) -> list:
    """The Rayleigh damping set: the piezo layer's elastic stiffness only, every other
    material zero (solver.py:111-113)."""
    return [mt.Material(m.rho, m.C, 0 * m.e, 0 * m.eps) if i == 0 else mt.Material(m.rho, 0 * m.C, 0 * m.e, 0 * m.eps)
            for i, m in enumerate(materials)]


def engine_for(case, loss: Loss, device: int = 0):
    """The GPU engine of ``case_for``'s result, with Rayleigh damping when the
    configuration asks for it (Q9 templates; the reference rejects loss on the
    Hex27 slabs)."""
    from .engine import FrequencySolver
    if isinstance(case, cases.HexCase):
        if loss.beta_dk:
            raise ValueError('Rayleigh damping is not defined for the Hex27 slabs')
        return cases.hex_engine_for(case, device=device)
    damping = damping_materials(case.materials) if loss.beta_dk else None
    return FrequencySolver.from_q9(case.mesh, case.materials, case.mat_idx, case.pml, case.omega_top, case.bc,
                                   mode_extension=case.mode_extension, damping_materials=damping,
                                   beta=loss.beta_dk, device=device)

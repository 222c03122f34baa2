"""ctypes signatures of the SemiSim 3D core ABI (the ``api3_*`` entry points).

The table restates the C signatures of the reference core (semiconductor_3d.c:4570-5353)
as main.py binds them (main.py:172-219, main.py:3490-3530, validate.py:31-53).  One table
serves every library that exports the ABI: the B200 solver library of this package and,
in the tests, the reference core built from source.

``bind(lib)`` sets ``restype``/``argtypes`` on every symbol the library exports and returns
the library, so calls such as ``lib.api3_set_contact_V(0, 0.6)`` convert their arguments.
"""
import ctypes

_I = ctypes.c_int
_D = ctypes.c_double
_LL = ctypes.c_longlong
_IP = ctypes.POINTER(ctypes.c_int)
_DP = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); the 89 entries of the reference core, in source order
API3 = {
    "api3_init": (None, []),                                              # C:4570
    "api3_set_threads": (None, [_I]),                                     # C:4599
    "api3_set_verbose": (None, [_I]),                                     # C:4607
    "api3_trap_species": (_I, [_I, _I, _D, _D, _D]),                      # C:4618
    "api3_trap_add": (_I, [_I, _I, _IP, _DP]),                            # C:4629
    "api3_traps_clear": (None, []),                                       # C:4645
    "api3_charge_add": (_I, [_I, _IP, _DP]),                              # C:4646
    "api3_n_trap_entries": (_I, []),                                      # C:4653
    "api3_set_models": (None, [_I]),                                      # C:4657
    "api3_set_caxis": (None, [_I]),                                       # C:4660
    "api3_get_caxis": (_I, []),                                           # C:4661
    "api3_add_material": (_I, [_I, _D]),                                  # C:4663
    "api3_set_mat_tau": (_I, [_I, _D, _D]),                               # C:4671
    "api3_set_grid_coords": (_I, [_I, _I, _I, _DP, _DP, _DP]),            # C:4679
    "api3_set_grid": (None, [_I, _I, _I, _D, _D, _D]),                    # C:4693
    "api3_set_solver": (None, [_I, _I, _I, _D, _D, _D, _D]),              # C:4708
    "api3_set_region": (None, [_I, _I, _I, _I, _I, _I, _I, _D, _D]),      # C:4718
    "api3_add_fixed_charge": (None, [_I, _I, _I, _I, _I, _I, _D]),        # C:4731
    "api3_add_sheet_charge": (None, [_I, _I, _I, _I, _I, _I, _D]),        # C:4742
    "api3_add_contact_ex": (_I, [_I] * 8 + [_D, _D, _D, _D]),             # C:4757
    "api3_add_contact": (None, [_I] * 6 + [_D, _D]),                      # C:4772
    "api3_clear_contacts": (None, []),                                    # C:4775
    "api3_set_gate_stack": (_I, [_I, _I, _IP, _DP]),                      # C:4779
    "api3_set_mesh_graph": (_I, [_I, _I, _IP, _IP, _DP, _DP, _DP, _DP]),  # C:4795
    "api3_is_graph": (_I, []),                                            # C:4806
    "api3_set_node_data": (None, [_IP, _DP, _DP, _DP]),                   # C:4808
    "api3_set_con_nodes": (_I, [_I, _I, _IP, _DP]),                       # C:4821
    "api3_set_walls": (None, [_DP]),                                      # C:4838
    "api3_get_ntp": (_I, [_I]),                                           # C:4844
    "api3_tun_eval": (_D, [_I, _I, _IP, _DP, _D, _D, _D, _D, _D, _DP]),   # C:4855
    "api3_mlda_factor": (_D, [_I, _D, _D, _I]),                           # C:4869
    "api3_coulomb_inv": (_D, [_I, _D, _D, _D, _D]),                       # C:4878
    "api3_set_surface_mobility": (_I, [_I, _D, _D, _D]),                  # C:4885
    "api3_lombardi": (_D, [_I, _D, _D, _D, _D, _I]),                      # C:4894
    "api3_set_contact_V": (None, [_I, _D]),                               # C:4898
    "api3_get_ncon": (_I, []),                                            # C:4899
    "api3_get_contact_I": (_D, [_I]),                                     # C:4900
    "api3_get_contact_A": (_D, [_I]),                                     # C:4901
    "api3_get_contact_In": (_D, [_I]),                                    # C:4902
    "api3_get_contact_Ifloor": (_D, [_I]),                                # C:4904
    "api3_get_contact_Iraw": (_D, [_I]),                                  # C:4906
    "api3_get_aa_depth": (_I, []),                                        # C:4907
    "api3_get_contact_Vsolved": (_D, [_I]),                               # C:4908
    "api3_request_stop": (None, []),                                      # C:4922
    "api3_clear_stop": (None, []),                                        # C:4923
    "api3_stop_requested": (_I, []),                                      # C:4924
    "api3_get_progress": (None, [_DP]),                                   # C:4926
    "api3_solve": (_I, []),                                               # C:4928
    "api3_resolve": (_I, []),                                             # C:4930
    "api3_iv_sweep": (None, [_I, _D, _D, _I, _DP, _DP, _IP]),             # C:4934
    "api3_iv_sweep2": (None, [_I, _D, _D, _I, _DP, _DP, _DP, _IP]),       # C:4958
    "api3_get_Emax": (_D, []),                                            # C:4981
    "api3_get_Nx": (_I, []),                                              # C:5003
    "api3_get_Ny": (_I, []),                                              # C:5004
    "api3_get_Nz": (_I, []),                                              # C:5005
    "api3_get_conv": (_I, []),                                            # C:5006
    "api3_get_iter": (_I, []),                                            # C:5007
    "api3_get_res": (_D, []),                                             # C:5008
    "api3_get_xs": (_D, [_I]),                                            # C:5009
    "api3_get_ys": (_D, [_I]),                                            # C:5010
    "api3_get_zs": (_D, [_I]),                                            # C:5011
    "api3_get_Cref": (_D, []),                                            # C:5012
    "api3_get_stat": (_LL, [_I]),                                         # C:5013
    "api3_set_predictor": (None, [_I]),                                   # C:5019
    "api3_get_state": (_I, [_DP, _DP, _DP]),                              # C:5023
    "api3_set_state": (_I, [_DP, _DP, _DP]),                              # C:5030
    "api3_get_time": (_D, [_I]),                                          # C:5043
    "api3_mat_ni": (_D, [_I]),                                            # C:5048
    "api3_mat_Eg": (_D, [_I]),                                            # C:5049
    "api3_bulk_copy": (None, [_I, _DP]),                                  # C:5127
    "api3_carrier_sums": (None, [_DP]),                                   # C:5137
    "api3_charge_partition": (_I, [_IP]),                                 # C:5192
    "api3_terminal_charges": (_I, [_I, _DP]),                             # C:5248
    "api3_face_J": (_I, [_I, _I, _DP]),                                   # C:5284
    "api3_charge_owner": (_I, [_IP]),                                     # C:5300
    "api3_ins_field_max": (_D, [_DP]),                                    # C:5308
    "api3_get_phi": (_D, [_I]),                                           # C:5341
    "api3_get_n": (_D, [_I]),                                             # C:5342
    "api3_get_p": (_D, [_I]),                                             # C:5343
    "api3_get_Ec": (_D, [_I]),                                            # C:5344
    "api3_get_Ev": (_D, [_I]),                                            # C:5345
    "api3_get_Efn": (_D, [_I]),                                           # C:5346
    "api3_get_Efp": (_D, [_I]),                                           # C:5347
    "api3_get_Jx": (_D, [_I]),                                            # C:5348
    "api3_get_Jy": (_D, [_I]),                                            # C:5349
    "api3_get_Jz": (_D, [_I]),                                            # C:5350
    "api3_get_mun": (_D, [_I]),                                           # C:5351
    "api3_get_mup": (_D, [_I]),                                           # C:5352
    "api3_get_R": (_D, [_I]),                                             # C:5353
}

# additive entries that both the B200 library and the oracle harness export
EXTRA = {
    # constant low-field mobility (m^2/Vs) of a material; no reference counterpart
    "api3_set_mat_mobility": (_I, [_I, _D, _D]),
    # more solver instances (the reference has one global device); per-thread selection
    "api3b_new": (_I, []),
    "api3b_use": (_I, [_I]),
    "api3b_current": (_I, []),
    "api3b_free": (_I, [_I]),
    # linear-solve precision of the current instance (0 FP64, 1 FP32 refined in FP64)
    "api3b_set_precision": (_I, [_I]),
    "api3b_get_precision": (_I, []),
    "api3b_set_persist": (_I, [_I, _I]),
    "api3b_set_share": (_I, [_I]),
    "api3b_set_pred_order": (_I, [_I]),
    # learned sweep predictor of the current instance
    "api3b_seed_set_model": (_I, [ctypes.POINTER(ctypes.c_float), _I]),
    "api3b_seed_enable": (_I, [_I]),
    "api3b_seed_stats": (None, [ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "api3b_seed_nparam": (_I, []),
    # launch-shape autotuner of the current instance
    "api3b_autotune": (_D, [_I]),
    # batched resolve of several bias vectors from the current solved state
    "api3b_resolve_batch": (_I, [_I, ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_D), ctypes.POINTER(_I), _I]),
    "api3b_resolve_batch_free": (_I, []),
    "api3b_tune_get": (_I, [ctypes.POINTER(_I)] * 4),
}


def bind(lib, table=None):
    """Declare the signatures of every table entry ``lib`` exports; returns ``lib``."""
    tab = dict(API3)
    tab.update(EXTRA)
    if table:
        tab.update(table)
    for name, (res, args) in tab.items():
        f = getattr(lib, name, None)
        if f is None:
            continue
        f.restype = res
        f.argtypes = args
    return lib


def dptr(a):
    """ctypes double* of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_DP)


def iptr(a):
    """ctypes int* of a C-contiguous int32 numpy array."""
    return a.ctypes.data_as(_IP)

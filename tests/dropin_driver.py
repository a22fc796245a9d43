"""mat_mult's partition loop (src/multiply_module.f90:115-359) driving the drop-in kernel pair.

This is the call sequence a Fortran build with MULT_KERN=gpu would make: for
every A-halo partition, copy the B partition's index block and data
(Mquest_get_local), build ibpart_rem (end_part_comms) and call m_kern_max /
m_kern_min with the reference argument lists.  The index arrays come from the
oracle's export (the reference layout).
"""
import numpy as np

import cq_b200


def _loc_trans(o, r, a, atrans, invdir):
    """loc_trans (multiply_module.f90:454-539)."""
    nh = int(o.geti("halo_sizes", r)[1])
    ndimj = o.geti("halo_ndimj", r)
    ndimi = o.geti("ndimi", r)
    i_h2d = o.geti("i_h2d", r)
    t_prim, t_beg, t_ndb, t_n = o.geti("t_i_prim", r), o.geti("t_i_beg", r), o.geti("t_i_nd_beg", r), o.geti("t_n_hnab", r)
    for ni in range(1, nh + 1):
        tpos = t_ndb[ni - 1]
        nd2 = ndimj[ni - 1]
        for nn in range(1, t_n[ni - 1] + 1):
            i = t_prim[t_beg[ni - 1] + nn - 2]
            istart = i_h2d[(i - 1) * nh + ni - 1]
            nd1 = ndimi[i - 1]
            blk = a[istart - 1:istart - 1 + nd1 * nd2].reshape(nd2, nd1)       # a(n1 + nd1*n2)
            if invdir == 0:
                atrans[tpos - 1:tpos - 1 + nd1 * nd2] = blk.ravel(order="F")   # atrans(n2 + nd2*n1)
            else:
                a[istart - 1:istart - 1 + nd1 * nd2] = atrans[tpos - 1:tpos - 1 + nd1 * nd2].reshape(nd1, nd2).ravel(order="F")
            tpos += nd1 * nd2


def mat_mult_dropin(o, mult_type, ra, rb, rc, a, b, c, deferred=False):
    """deferred: the shim passes ahalo%np_in_halo before every call (cq_m_kern_defer), so the loop's calls
    enqueue their work and the last partition's call completes it."""
    cd = o.geti("cover_dims")
    ncy, ncz = int(cd[1]), int(cd[2])
    ngnode = o.geti("ngnode")
    i_cc2seq = np.zeros(len(ngnode) + 1, np.int64)
    i_cc2seq[ngnode] = np.arange(1, len(ngnode) + 1)
    nm_group = o.geti("nm_group")
    # A halo + retro of range ra, C halo of range rc
    ah = dict(nh_part=o.geti("nh_part", ra), j_beg=o.geti("j_beg", ra), j_seq=o.geti("j_seq", ra),
              ndimi=o.geti("ndimi", ra), ndimj=o.geti("halo_ndimj", ra))
    lab_hcell, lab_hcover = o.geti("lab_hcell", ra), o.geti("lab_hcover", ra)
    at = dict(i_prim=o.geti("t_i_prim", ra), i_beg=o.geti("t_i_beg", ra), i_nd_beg=o.geti("t_i_nd_beg", ra),
              n_hnab=o.geti("t_n_hnab", ra))
    ch = dict(i_halo=o.geti("i_halo", rc), i_hbeg=o.geti("i_hbeg", rc), i_h2d=o.geti("i_h2d", rc),
              ni_in_halo=int(o.geti("halo_sizes", rc)[1]))
    # B index of range rb
    bind = o.geti("bind", rb)
    posn = o.geti("array_posn", rb)
    nnab_b = o.geti("n_nab", rb)
    ndimi_b = o.geti("ndimi", rb)
    ndimj_b = o.geti("ndimj", rb)
    i_nd_acc_b = o.geti("i_nd_acc", rb)
    nm_nod = o.geti("nm_nodgroup")
    first_atom = np.concatenate([[0], np.cumsum(nm_nod)])
    first_blk = np.concatenate([[0], np.cumsum(nnab_b)])
    lena = a.size
    atrans = np.zeros(lena)
    if mult_type == 1:
        _loc_trans(o, ra, a, atrans, 0)
        c[:] = 0.0
    for kpart in range(1, len(lab_hcell) + 1):
        ind_part = lab_hcell[kpart - 1]
        ipart = int(i_cc2seq[ind_part])
        n_cont = int(nm_group[ind_part - 1])
        p0, p1 = first_atom[ipart - 1], first_atom[ipart]
        part_nabs = int(nnab_b[p0:p1].sum())
        e0, e1 = first_blk[p0], first_blk[p1]
        part_nd_nabs = int((ndimi_b[np.repeat(np.arange(p0, p1), nnab_b[p0:p1])] * ndimj_b[e0:e1]).sum())
        indsize = 3 * n_cont + 5 * part_nabs
        pa = bind[posn[ipart - 1] - 1:posn[ipart - 1] - 1 + indsize]
        nd_off = int(i_nd_acc_b[p0]) - 1
        b_rem = np.ascontiguousarray(b[nd_off:nd_off + part_nd_nabs])
        nbnab, ibind, ib_nd_acc = pa[:n_cont], pa[n_cont:2 * n_cont], pa[2 * n_cont:3 * n_cont]
        ibseq = pa[3 * n_cont:3 * n_cont + part_nabs]
        npxyz = pa[3 * n_cont + part_nabs:3 * n_cont + 4 * part_nabs]
        bndim2 = pa[3 * n_cont + 4 * part_nabs:3 * n_cont + 5 * part_nabs]
        ibpart = np.zeros(part_nabs, np.int64)   # end_part_comms
        noff = 0
        for k in range(n_cont):
            for ni in range(nbnab[k]):
                ibpart[ibind[k] + ni - 1] = npxyz[noff + 3 * ni] * ncy * ncz + npxyz[noff + 3 * ni + 1] * ncz + npxyz[noff + 3 * ni + 2]
            noff += 3 * nbnab[k]
        k_off = int(lab_hcover[kpart - 1])
        if deferred:
            cq_b200.m_kern_defer(len(lab_hcell))
        cq_b200.m_kern("max" if mult_type == 1 else "min", k_off, kpart, ib_nd_acc, ibind, nbnab, ibpart, ibseq, bndim2,
                       atrans, b_rem, c, ah, ch, at)
    if deferred:
        cq_b200.m_kern_defer(0)
    if mult_type == 2:
        _loc_trans(o, ra, a, atrans, 1)

/*
 * CPU oracle: region topology, halo/pole communication lists and the data
 * transfer, restated from the reference "communication" kernel.
 * TEST INFRASTRUCTURE ONLY (see icoadv_oracle.h).
 *
 *   ADM_setup sizes              communication/src/mod_adm.f90:220-251
 *   RGNMNG_generate_ico          communication/src/mod_adm.f90:629-804
 *   RGNMNG_vertex_walkaround     communication/src/mod_adm.f90:808-894
 *   rgn4pl / ADM_have_sgp        communication/src/mod_adm.f90:257-265,393-406
 *   COMM_list_generate           communication/src/mod_comm.f90:213-609
 *   COMM_sortdest                communication/src/mod_comm.f90:613-920
 *   COMM_sortdest_pl             communication/src/mod_comm.f90:924-1380
 *   COMM_sortdest_singular       communication/src/mod_comm.f90:1384-1502
 *   COMM_data_transfer           communication/src/mod_comm.f90:1506-1891
 *   COMM_var                     communication/src/mod_comm.f90:1895-2101
 *
 * MPI is emulated in one address space: every rank's lists are built exactly
 * as the reference builds them (including the allgather ordering of the
 * send-side tables), and a transfer packs every rank's send buffers in its
 * Send_list order before the local copies, then unpacks in the receiver's
 * Recv_list order after them, which is the order MPI imposes.  This is what
 * reproduces the reference's 2-rank golden logs bit for bit, including the
 * order in which r2p values land in the south-pole ring.
 */
#include "icoadv_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { I_SW = 1, I_NW, I_NE, I_SE };
enum { I_W = 1, I_N, I_E, I_S };
enum { I_NPL = 1, I_SPL = 2 };
#define VLINK 5
#define MAXPEER 10 /* Recv_nlim / Send_nlim, mod_comm.f90:111-112 */

typedef struct {
  int n, cap;
  int *e; /* 4 ints per entry: grid_from, l_from, grid_to, l_to (1-based) */
} lst;

typedef struct {
  int size, prc_from, prc_to;
  lst list;
} peer;

typedef struct {
  lst rel; /* rellist: 6 ints per entry */
  lst copy_r2r, copy_p2r, copy_r2p, singular;
  int nrecv_r2r, nsend_r2r, nrecv_p2r, nsend_p2r, nrecv_r2p, nsend_r2p;
  peer recv_r2r[MAXPEER], send_r2r[MAXPEER];
  peer recv_p2r[MAXPEER], send_p2r[MAXPEER];
  peer recv_r2p[MAXPEER], send_r2p[MAXPEER];
} rank_state;

struct orc_topo {
  int glevel, rlevel, nprocs;
  int rgn_nmax, lall, gall_1d, gall, gmin, gmax;
  int *edge_tab; /* [rgn][4][2]  (rgnid, dir) */
  int *vert_num; /* [rgn][4] */
  int *vert_tab; /* [rgn][4][VLINK][2] */
  int vert_tab_pl[3][VLINK + 1][2];
  int rgn4pl[3];
  int r2p_pl[3];
  int *lp2r; /* [p][l] p,l 1-based, stored (p-1)*lall + (l-1) */
  int *r2lp; /* [rgn][2] (l, prc) */
  rank_state *rk;
};

static void lst_push(lst *L, int width, const int *v) {
  if (L->n == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 64;
    L->e = realloc(L->e, sizeof(int) * width * L->cap);
  }
  memcpy(L->e + (size_t)width * L->n, v, sizeof(int) * width);
  L->n++;
}

#define ET(t, r, d, x) (t)->edge_tab[(((r)-1) * 4 + ((d)-1)) * 2 + (x)]
#define VN(t, r, d) (t)->vert_num[((r)-1) * 4 + ((d)-1)]
#define VT(t, r, d, v, x) (t)->vert_tab[((((r)-1) * 4 + ((d)-1)) * VLINK + ((v)-1)) * 2 + (x)]
#define LP2R(t, l, p) (t)->lp2r[((p)-1) * (t)->lall + ((l)-1)]
#define R2L(t, r) (t)->r2lp[((r)-1) * 2 + 0]
#define R2P(t, r) (t)->r2lp[((r)-1) * 2 + 1]

static int suf(const orc_topo *t, int i, int j) { return t->gall_1d * (j - 1) + i; }

static void generate_ico(orc_topo *t) {
  static const int dmd_data[11][5] = {{0},
      {0, 6, 5, 2, 10}, {0, 10, 1, 3, 9}, {0, 9, 2, 4, 8}, {0, 8, 3, 5, 7}, {0, 7, 4, 1, 6},
      {0, 7, 5, 1, 10}, {0, 8, 4, 5, 6}, {0, 9, 3, 4, 7}, {0, 10, 2, 3, 8}, {0, 6, 1, 2, 9}};
  int rall_1d = 1 << t->rlevel, rall_1dmd = rall_1d * rall_1d;
  for (int d = 1; d <= 10; ++d)
    for (int i = 1; i <= rall_1d; ++i)
      for (int j = 1; j <= rall_1d; ++j) {
        int rgnid = (d - 1) * rall_1dmd + (j - 1) * rall_1d + i;
        int i_nb, j_nb, d_nb, dir;
        /* SW */
        if (j == 1) {
          if (d <= 5) { i_nb = i; j_nb = rall_1d; d_nb = dmd_data[d][I_SW]; dir = I_NE; }
          else { i_nb = rall_1d; j_nb = rall_1d + 1 - i; d_nb = dmd_data[d][I_SW]; dir = I_SE; }
        } else { i_nb = i; j_nb = j - 1; d_nb = d; dir = I_NE; }
        ET(t, rgnid, I_SW, 0) = (d_nb - 1) * rall_1dmd + (j_nb - 1) * rall_1d + i_nb;
        ET(t, rgnid, I_SW, 1) = dir;
        /* NW */
        if (i == 1) {
          if (d <= 5) { i_nb = rall_1d + 1 - j; j_nb = rall_1d; d_nb = dmd_data[d][I_NW]; dir = I_NE; }
          else { i_nb = rall_1d; j_nb = j; d_nb = dmd_data[d][I_NW]; dir = I_SE; }
        } else { i_nb = i - 1; j_nb = j; d_nb = d; dir = I_SE; }
        ET(t, rgnid, I_NW, 0) = (d_nb - 1) * rall_1dmd + (j_nb - 1) * rall_1d + i_nb;
        ET(t, rgnid, I_NW, 1) = dir;
        /* NE */
        if (j == rall_1d) {
          if (d <= 5) { i_nb = 1; j_nb = rall_1d + 1 - i; d_nb = dmd_data[d][I_NE]; dir = I_NW; }
          else { i_nb = i; j_nb = 1; d_nb = dmd_data[d][I_NE]; dir = I_SW; }
        } else { i_nb = i; j_nb = j + 1; d_nb = d; dir = I_SW; }
        ET(t, rgnid, I_NE, 0) = (d_nb - 1) * rall_1dmd + (j_nb - 1) * rall_1d + i_nb;
        ET(t, rgnid, I_NE, 1) = dir;
        /* SE */
        if (i == rall_1d) {
          if (d <= 5) { i_nb = 1; j_nb = j; d_nb = dmd_data[d][I_SE]; dir = I_NW; }
          else { i_nb = rall_1d + 1 - j; j_nb = 1; d_nb = dmd_data[d][I_SE]; dir = I_SW; }
        } else { i_nb = i + 1; j_nb = j; d_nb = d; dir = I_NW; }
        ET(t, rgnid, I_SE, 0) = (d_nb - 1) * rall_1dmd + (j_nb - 1) * rall_1d + i_nb;
        ET(t, rgnid, I_SE, 1) = dir;
      }
}

static void vertex_walkaround(orc_topo *t) {
  for (int i = 0; i < t->rgn_nmax * 4; ++i) t->vert_num[i] = -1;
  for (int i = 0; i < t->rgn_nmax * 4 * VLINK * 2; ++i) t->vert_tab[i] = -1;
  for (int r = 1; r <= t->rgn_nmax; ++r)
    for (int d = I_W; d <= I_S; ++d) {
      int rgnid = r;
      int dir = (d == I_W) ? I_SW : (d == I_N) ? I_NW : (d == I_E) ? I_NE : I_SE;
      int v = 0;
      for (;;) {
        int rgnid_next = ET(t, rgnid, dir, 0);
        int dir_next = ET(t, rgnid, dir, 1) - 1;
        if (dir_next == 0) dir_next = 4;
        v = v + 1;
        VT(t, r, d, v, 0) = rgnid;
        VT(t, r, d, v, 1) = dir;
        rgnid = rgnid_next;
        dir = dir_next;
        if (rgnid == r) break;
      }
      VN(t, r, d) = v;
    }
  for (int p = 0; p < 3; ++p)
    for (int v = 0; v <= VLINK; ++v) t->vert_tab_pl[p][v][0] = t->vert_tab_pl[p][v][1] = -1;
  for (int r = 1; r <= t->rgn_nmax; ++r)
    if (VN(t, r, I_N) == VLINK) {
      for (int v = 1; v <= VLINK; ++v) {
        t->vert_tab_pl[I_NPL][v][0] = VT(t, r, I_N, v, 0);
        t->vert_tab_pl[I_NPL][v][1] = VT(t, r, I_N, v, 1);
      }
      break;
    }
  for (int r = 1; r <= t->rgn_nmax; ++r)
    if (VN(t, r, I_S) == VLINK) {
      for (int v = 1; v <= VLINK; ++v) {
        t->vert_tab_pl[I_SPL][v][0] = VT(t, r, I_S, v, 0);
        t->vert_tab_pl[I_SPL][v][1] = VT(t, r, I_S, v, 1);
      }
      break;
    }
}

/* COMM_list_generate for rank prc (mod_comm.f90:213-609) */
static void list_generate(orc_topo *t, int prc) {
  rank_state *R = &t->rk[prc - 1];
  int gmin = t->gmin, gmax = t->gmax, ginnar = gmax - gmin + 1;
  for (int l = 1; l <= t->lall; ++l) {
    int rgnid = LP2R(t, l, prc);
    int e[6];
#define PUSH(ii, jj, ir, jr)                                                   \
  do {                                                                         \
    e[0] = suf(t, ii, jj); e[1] = rgnid; e[2] = prc;                           \
    e[3] = suf(t, ir, jr); e[4] = rgnid_rmt; e[5] = prc_rmt;                   \
    lst_push(&R->rel, 6, e);                                                   \
  } while (0)
    int rgnid_rmt, prc_rmt;
    /* South West */
    if (ET(t, rgnid, I_SW, 1) == I_NE) {
      rgnid_rmt = ET(t, rgnid, I_SW, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin - 1 + n, gmin - 1, gmin - 1 + n, gmax);
    }
    if (ET(t, rgnid, I_SW, 1) == I_SE) {
      rgnid_rmt = ET(t, rgnid, I_SW, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin - 1 + n, gmin - 1, gmax, gmax + 1 - n);
    }
    /* North West */
    if (ET(t, rgnid, I_NW, 1) == I_SE) {
      rgnid_rmt = ET(t, rgnid, I_NW, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin - 1, gmin - 1 + n, gmax, gmin - 1 + n);
    }
    if (ET(t, rgnid, I_NW, 1) == I_NE) {
      rgnid_rmt = ET(t, rgnid, I_NW, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin - 1, gmin - 1 + n, gmax + 1 - n, gmax);
    }
    /* North East */
    if (ET(t, rgnid, I_NE, 1) == I_SW) {
      rgnid_rmt = ET(t, rgnid, I_NE, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin - 1 + n, gmax + 1, gmin - 1 + n, gmin);
    }
    if (ET(t, rgnid, I_NE, 1) == I_NW) {
      rgnid_rmt = ET(t, rgnid, I_NE, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmin + n, gmax + 1, gmin, gmax + 1 - n);
    }
    /* South East */
    if (ET(t, rgnid, I_SE, 1) == I_NW) {
      rgnid_rmt = ET(t, rgnid, I_SE, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmax + 1, gmin - 1 + n, gmin, gmin - 1 + n);
    }
    if (ET(t, rgnid, I_SE, 1) == I_SW) {
      rgnid_rmt = ET(t, rgnid, I_SE, 0); prc_rmt = R2P(t, rgnid_rmt);
      for (int n = 1; n <= ginnar; ++n) PUSH(gmax + 1, gmin + n, gmax + 1 - n, gmin);
    }
    /* Vertex links */
    if (VN(t, rgnid, I_W) == 4) {
      rgnid_rmt = VT(t, rgnid, I_W, 3, 0); prc_rmt = R2P(t, rgnid_rmt);
      int dv = VT(t, rgnid, I_W, 3, 1), ir = -1, jr = -1;
      if (dv == I_N) { ir = gmin; jr = gmax; }
      else if (dv == I_E) { ir = gmax; jr = gmax; }
      else if (dv == I_S) { ir = gmax; jr = gmin; }
      PUSH(gmin - 1, gmin - 1, ir, jr);
    }
    if (VN(t, rgnid, I_N) == 4) {
      rgnid_rmt = VT(t, rgnid, I_N, 3, 0); prc_rmt = R2P(t, rgnid_rmt);
      int dv = VT(t, rgnid, I_N, 3, 1), ir = -1, jr = -1;
      if (dv == I_W) PUSH(gmin, gmax + 1, gmin, gmin);
      if (dv == I_W) { ir = gmin; jr = gmin + 1; }
      else if (dv == I_N) { ir = gmin; jr = gmax; }
      else if (dv == I_E) { ir = gmax; jr = gmax; }
      else if (dv == I_S) { ir = gmax; jr = gmin; }
      PUSH(gmin - 1, gmax + 1, ir, jr);
    }
    if (VN(t, rgnid, I_E) == 4) {
      if (VT(t, rgnid, I_E, 3, 1) == I_W) {
        rgnid_rmt = VT(t, rgnid, I_E, 3, 0); prc_rmt = R2P(t, rgnid_rmt);
        PUSH(gmax + 1, gmax + 1, gmin, gmin);
      }
    }
    if (VN(t, rgnid, I_S) == 4) {
      rgnid_rmt = VT(t, rgnid, I_S, 3, 0); prc_rmt = R2P(t, rgnid_rmt);
      int dv = VT(t, rgnid, I_S, 3, 1), ir = -1, jr = -1;
      if (dv == I_W) PUSH(gmax + 1, gmin, gmin, gmin);
      if (dv == I_W) { ir = gmin + 1; jr = gmin; }
      else if (dv == I_N) { ir = gmin; jr = gmax; }
      else if (dv == I_E) { ir = gmax; jr = gmax; }
      else if (dv == I_S) { ir = gmax; jr = gmin; }
      PUSH(gmax + 1, gmin - 1, ir, jr);
    }
#undef PUSH
  }
}

static peer *find_peer(peer *P, int *n, int key_from, int key_to, int match_from) {
  for (int i = 0; i < *n; ++i)
    if ((match_from ? P[i].prc_from : P[i].prc_to) == (match_from ? key_from : key_to)) return &P[i];
  peer *p = &P[(*n)++];
  memset(p, 0, sizeof(*p));
  p->prc_from = key_from;
  p->prc_to = key_to;
  return p;
}

/* COMM_sortdest (mod_comm.f90:613-920), all ranks at once (the MPI_Allgather
 * and the list exchange become reads of the other ranks' tables). */
static void sortdest(orc_topo *t) {
  for (int p = 1; p <= t->nprocs; ++p) {
    rank_state *R = &t->rk[p - 1];
    for (int c = 0; c < R->rel.n; ++c) {
      const int *r = R->rel.e + 6 * c;
      int e[4] = {r[3], R2L(t, r[4]), r[0], R2L(t, r[1])};
      if (r[2] == r[5]) {
        lst_push(&R->copy_r2r, 4, e);
      } else {
        peer *pp = find_peer(R->recv_r2r, &R->nrecv_r2r, r[5], r[2], 1);
        pp->size++;
        lst_push(&pp->list, 4, e);
      }
    }
  }
  int nglobal = 0;
  for (int p = 1; p <= t->nprocs; ++p)
    if (t->rk[p - 1].nrecv_r2r > nglobal) nglobal = t->rk[p - 1].nrecv_r2r;
  /* recvbuf_info: rank order, nglobal slots each; accept requests to me */
  for (int me = 1; me <= t->nprocs; ++me) {
    rank_state *S = &t->rk[me - 1];
    for (int p = 1; p <= t->nprocs; ++p) {
      rank_state *R = &t->rk[p - 1];
      for (int ir = 0; ir < nglobal && ir < R->nrecv_r2r; ++ir) {
        if (R->recv_r2r[ir].prc_from == me) {
          peer *s = &S->send_r2r[S->nsend_r2r++];
          memset(s, 0, sizeof(*s));
          s->size = R->recv_r2r[ir].size;
          s->prc_from = R->recv_r2r[ir].prc_from;
          s->prc_to = R->recv_r2r[ir].prc_to;
          for (int i = 0; i < R->recv_r2r[ir].list.n; ++i) lst_push(&s->list, 4, R->recv_r2r[ir].list.e + 4 * i);
        }
      }
    }
  }
}

/* COMM_sortdest_pl (mod_comm.f90:924-1380) */
static void sortdest_pl(orc_topo *t) {
  int gmin = t->gmin, gmax = t->gmax;
  for (int prc = 1; prc <= t->nprocs; ++prc) {
    rank_state *R = &t->rk[prc - 1];
    for (int l = 1; l <= t->lall; ++l) {
      int rgnid = LP2R(t, l, prc);
      for (int l_pl = I_NPL; l_pl <= I_SPL; ++l_pl) {
        int rgnid_rmt = l_pl, prc_rmt = t->r2p_pl[rgnid_rmt];
        int check, i_from, j_from, i_to, j_to;
        if (rgnid_rmt == I_NPL) { check = VN(t, rgnid, I_N); i_from = gmin; j_from = gmax; i_to = gmin; j_to = gmax + 1; }
        else { check = VN(t, rgnid, I_S); i_from = gmax; j_from = gmin; i_to = gmax + 1; j_to = gmin; }
        if (check == VLINK) {
          int pl_to = -1;
          for (int v = 1; v <= VLINK; ++v)
            if (rgnid == t->vert_tab_pl[rgnid_rmt][v][0]) {
              pl_to = v;
              if (pl_to < 2) pl_to = 6;
              break;
            }
          if (prc == prc_rmt) {
            int e[4] = {suf(t, i_from, j_from), l, pl_to, l_pl};
            lst_push(&R->copy_r2p, 4, e);
          } else {
            peer *pp = find_peer(R->recv_p2r, &R->nrecv_p2r, prc_rmt, prc, 1);
            pp->size++;
            int e1[4] = {1, l_pl, suf(t, i_to, j_to), l};
            lst_push(&pp->list, 4, e1);
            pp = find_peer(R->send_r2p, &R->nsend_r2p, prc, prc_rmt, 0);
            pp->size++;
            int e2[4] = {suf(t, i_from, j_from), l, pl_to, l_pl};
            lst_push(&pp->list, 4, e2);
          }
        }
      }
    }
    if (prc == t->r2p_pl[I_NPL]) { /* ADM_have_pl: the pole process */
      for (int l_pl = I_NPL; l_pl <= I_SPL; ++l_pl) {
        int rgnid = l_pl;
        for (int v = VLINK; v >= 1; --v) {
          int rgnid_rmt = t->vert_tab_pl[rgnid][v][0], prc_rmt = R2P(t, rgnid_rmt);
          int i_from, j_from, i_to, j_to;
          if (rgnid == I_NPL) { i_from = gmin; j_from = gmax; i_to = gmin; j_to = gmax + 1; }
          else { i_from = gmax; j_from = gmin; i_to = gmax + 1; j_to = gmin; }
          int pl_to = v;
          if (pl_to < 2) pl_to = 6;
          if (prc == prc_rmt) {
            int e[4] = {1, l_pl, suf(t, i_to, j_to), R2L(t, rgnid_rmt)};
            lst_push(&R->copy_p2r, 4, e);
          } else {
            peer *pp = find_peer(R->recv_r2p, &R->nrecv_r2p, prc_rmt, prc, 1);
            pp->size++;
            int e1[4] = {suf(t, i_from, j_from), R2L(t, rgnid_rmt), pl_to, l_pl};
            lst_push(&pp->list, 4, e1);
            pp = find_peer(R->send_p2r, &R->nsend_p2r, prc, prc_rmt, 0);
            pp->size++;
            int e2[4] = {1, l_pl, suf(t, i_to, j_to), R2L(t, rgnid_rmt)};
            lst_push(&pp->list, 4, e2);
          }
        }
      }
    }
  }
}

/* COMM_sortdest_singular (mod_comm.f90:1384-1502) */
static void sortdest_singular(orc_topo *t) {
  int gmin = t->gmin, gmax = t->gmax;
  for (int prc = 1; prc <= t->nprocs; ++prc) {
    rank_state *R = &t->rk[prc - 1];
    for (int l = 1; l <= t->lall; ++l) {
      int rgnid = LP2R(t, l, prc);
      if (VN(t, rgnid, I_W) == 3) {
        int e[4] = {suf(t, gmin, gmin - 1), l, suf(t, gmin - 1, gmin - 1), l};
        lst_push(&R->singular, 4, e);
      }
      if (VN(t, rgnid, I_N) != 4) {
        int e[4] = {suf(t, gmin - 1, gmax), l, suf(t, gmin - 1, gmax + 1), l};
        lst_push(&R->singular, 4, e);
      }
      if (VN(t, rgnid, I_S) != 4) {
        int e[4] = {suf(t, gmax + 1, gmin), l, suf(t, gmax + 1, gmin - 1), l};
        lst_push(&R->singular, 4, e);
      }
    }
  }
}

orc_topo *orc_topo_create(int glevel, int rlevel, int nprocs) {
  orc_topo *t = calloc(1, sizeof(*t));
  t->glevel = glevel;
  t->rlevel = rlevel;
  t->nprocs = nprocs;
  t->rgn_nmax = (1 << rlevel) * (1 << rlevel) * 10;
  if (t->rgn_nmax % nprocs) { free(t); return NULL; }
  t->lall = t->rgn_nmax / nprocs;
  int nmax = 1 << (glevel - rlevel);
  t->gall_1d = nmax + 2;
  t->gall = t->gall_1d * t->gall_1d;
  t->gmin = 2;
  t->gmax = nmax + 1;
  t->edge_tab = calloc((size_t)t->rgn_nmax * 8, sizeof(int));
  t->vert_num = calloc((size_t)t->rgn_nmax * 4, sizeof(int));
  t->vert_tab = calloc((size_t)t->rgn_nmax * 4 * VLINK * 2, sizeof(int));
  generate_ico(t);
  t->lp2r = calloc((size_t)nprocs * t->lall, sizeof(int));
  t->r2lp = calloc((size_t)t->rgn_nmax * 2, sizeof(int));
  int rgnid = 0;
  for (int p = 1; p <= nprocs; ++p)
    for (int l = 1; l <= t->lall; ++l) {
      rgnid++;
      LP2R(t, l, p) = rgnid;
      R2L(t, rgnid) = l;
      R2P(t, rgnid) = p;
    }
  vertex_walkaround(t);
  for (int r = 1; r <= t->rgn_nmax; ++r)
    if (VN(t, r, I_N) == VLINK) { t->rgn4pl[I_NPL] = r; break; }
  for (int r = 1; r <= t->rgn_nmax; ++r)
    if (VN(t, r, I_S) == VLINK) { t->rgn4pl[I_SPL] = r; break; }
  t->r2p_pl[I_NPL] = 1; /* ADM_prc_pl = 1, mod_adm.f90:190,408-409 */
  t->r2p_pl[I_SPL] = 1;
  t->rk = calloc(nprocs, sizeof(rank_state));
  for (int p = 1; p <= nprocs; ++p) list_generate(t, p);
  sortdest(t);
  sortdest_pl(t);
  sortdest_singular(t);
  return t;
}

static void lst_free(lst *L) { free(L->e); }

void orc_topo_destroy(orc_topo *t) {
  if (!t) return;
  for (int p = 0; p < t->nprocs; ++p) {
    rank_state *R = &t->rk[p];
    lst_free(&R->rel); lst_free(&R->copy_r2r); lst_free(&R->copy_p2r);
    lst_free(&R->copy_r2p); lst_free(&R->singular);
    for (int i = 0; i < MAXPEER; ++i) {
      lst_free(&R->recv_r2r[i].list); lst_free(&R->send_r2r[i].list);
      lst_free(&R->recv_p2r[i].list); lst_free(&R->send_p2r[i].list);
      lst_free(&R->recv_r2p[i].list); lst_free(&R->send_r2p[i].list);
    }
  }
  free(t->rk); free(t->edge_tab); free(t->vert_num); free(t->vert_tab);
  free(t->lp2r); free(t->r2lp); free(t);
}

int orc_topo_lall(const orc_topo *t) { return t->lall; }
int orc_topo_rgn_nmax(const orc_topo *t) { return t->rgn_nmax; }
int orc_topo_have_sgp(const orc_topo *t, int rank, int l) { return VN(t, LP2R(t, l, rank), I_W) == 3; }
int orc_topo_rgnid(const orc_topo *t, int rank, int l) { return LP2R(t, l, rank); }
void orc_topo_edge_tab(const orc_topo *t, int *out) { memcpy(out, t->edge_tab, sizeof(int) * 8 * t->rgn_nmax); }
void orc_topo_vert_num(const orc_topo *t, int *out) { memcpy(out, t->vert_num, sizeof(int) * 4 * t->rgn_nmax); }
int orc_topo_rgn4pl(const orc_topo *t, int pole) { return t->rgn4pl[pole]; }
int orc_topo_rellist_nmax(const orc_topo *t, int rank) { return t->rk[rank - 1].rel.n; }

/* element accessors for one rank's var(gall,kmax,lall,vmax) / var_pl(6,kmax,2,vmax) */
#define VAR(base, g, k, l, v) base[((((size_t)(v)-1) * t->lall + ((l)-1)) * kmax + ((k)-1)) * t->gall + ((g)-1)]
#define VPL(base, g, k, l, v) base[((((size_t)(v)-1) * 2 + ((l)-1)) * kmax + ((k)-1)) * 6 + ((g)-1)]

static const peer *match_send(const peer *S, int n, int prc_to) {
  for (int i = 0; i < n; ++i)
    if (S[i].prc_to == prc_to) return &S[i];
  return NULL;
}

void orc_comm_data_transfer(const orc_topo *t, double **var, double **var_pl, int kmax, int vmax) {
  const int np = t->nprocs;
  /* pack: value snapshot of every send list entry, sender order (:1619-1728) */
  double ***pk = calloc(np, sizeof(double **));
  for (int s = 0; s < np; ++s) {
    const rank_state *S = &t->rk[s];
    int nb = S->nsend_p2r + S->nsend_r2p + S->nsend_r2r;
    pk[s] = calloc(nb ? nb : 1, sizeof(double *));
    int b = 0;
    for (int ir = 0; ir < S->nsend_p2r; ++ir, ++b) {
      const lst *L = &S->send_p2r[ir].list;
      pk[s][b] = malloc(sizeof(double) * (size_t)L->n * kmax * vmax + 8);
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i] = VPL(var_pl[s], L->e[4 * i], k, L->e[4 * i + 1], v);
    }
    for (int ir = 0; ir < S->nsend_r2p; ++ir, ++b) {
      const lst *L = &S->send_r2p[ir].list;
      pk[s][b] = malloc(sizeof(double) * (size_t)L->n * kmax * vmax + 8);
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i] = VAR(var[s], L->e[4 * i], k, L->e[4 * i + 1], v);
    }
    for (int ir = 0; ir < S->nsend_r2r; ++ir, ++b) {
      const lst *L = &S->send_r2r[ir].list;
      pk[s][b] = malloc(sizeof(double) * (size_t)L->n * kmax * vmax + 8);
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i] = VAR(var[s], L->e[4 * i], k, L->e[4 * i + 1], v);
    }
  }
  /* local copies p2r, r2p, r2r (:1730-1791) */
  for (int r = 0; r < np; ++r) {
    const rank_state *R = &t->rk[r];
    for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < R->copy_p2r.n; ++i) {
      const int *e = R->copy_p2r.e + 4 * i;
      VAR(var[r], e[2], k, e[3], v) = VPL(var_pl[r], e[0], k, e[1], v);
    }
    for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < R->copy_r2p.n; ++i) {
      const int *e = R->copy_r2p.e + 4 * i;
      VPL(var_pl[r], e[2], k, e[3], v) = VAR(var[r], e[0], k, e[1], v);
    }
    for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < R->copy_r2r.n; ++i) {
      const int *e = R->copy_r2r.e + 4 * i;
      VAR(var[r], e[2], k, e[3], v) = VAR(var[r], e[0], k, e[1], v);
    }
  }
  /* unpack p2r, r2p, r2r in the receiver's list order (:1799-1866) */
  for (int r = 0; r < np; ++r) {
    const rank_state *R = &t->rk[r];
    for (int ir = 0; ir < R->nrecv_p2r; ++ir) {
      int s = R->recv_p2r[ir].prc_from - 1;
      const rank_state *S = &t->rk[s];
      const peer *sp = match_send(S->send_p2r, S->nsend_p2r, r + 1);
      int b = (int)(sp - S->send_p2r);
      const lst *L = &R->recv_p2r[ir].list;
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        VAR(var[r], L->e[4 * i + 2], k, L->e[4 * i + 3], v) = pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i];
    }
    for (int ir = 0; ir < R->nrecv_r2p; ++ir) {
      int s = R->recv_r2p[ir].prc_from - 1;
      const rank_state *S = &t->rk[s];
      const peer *sp = match_send(S->send_r2p, S->nsend_r2p, r + 1);
      int b = S->nsend_p2r + (int)(sp - S->send_r2p);
      const lst *L = &R->recv_r2p[ir].list;
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        VPL(var_pl[r], L->e[4 * i + 2], k, L->e[4 * i + 3], v) = pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i];
    }
    for (int ir = 0; ir < R->nrecv_r2r; ++ir) {
      int s = R->recv_r2r[ir].prc_from - 1;
      const rank_state *S = &t->rk[s];
      const peer *sp = match_send(S->send_r2r, S->nsend_r2r, r + 1);
      int b = S->nsend_p2r + S->nsend_r2p + (int)(sp - S->send_r2r);
      const lst *L = &R->recv_r2r[ir].list;
      for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < L->n; ++i)
        VAR(var[r], L->e[4 * i + 2], k, L->e[4 * i + 3], v) = pk[s][b][((size_t)(v - 1) * kmax + (k - 1)) * L->n + i];
    }
  }
  /* singular points, halo to halo (:1868-1884) */
  for (int r = 0; r < np; ++r) {
    const rank_state *R = &t->rk[r];
    for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k) for (int i = 0; i < R->singular.n; ++i) {
      const int *e = R->singular.e + 4 * i;
      VAR(var[r], e[2], k, e[3], v) = VAR(var[r], e[0], k, e[1], v);
    }
  }
  for (int s = 0; s < np; ++s) {
    const rank_state *S = &t->rk[s];
    int nb = S->nsend_p2r + S->nsend_r2p + S->nsend_r2r;
    for (int b = 0; b < nb; ++b) free(pk[s][b]);
    free(pk[s]);
  }
  free(pk);
}

void orc_comm_var(const orc_topo *t, double **var, double **var_pl, int kmax, int vmax) {
  /* p2r-reverse: pole centre <- halo point of rgn4pl (mod_comm.f90:1943-2092).
   * Every branch (recv/send/copy) moves var(grid_to of the p2r entry, l_to)
   * of region rgn4pl into var_pl(gslf_pl, l_pl) on the pole process. */
  int pole_rank = t->r2p_pl[I_NPL] - 1;
  for (int r = 0; r < t->nprocs; ++r) {
    const rank_state *R = &t->rk[r];
    /* region side entries: Recv_list_p2r (remote) or, on the pole rank, Copy_list_p2r */
    for (int ir = 0; ir < R->nrecv_p2r; ++ir) {
      const lst *L = &R->recv_p2r[ir].list;
      for (int i = 0; i < L->n; ++i) {
        const int *e = L->e + 4 * i;
        int r_from = LP2R(t, e[3], R->recv_p2r[ir].prc_to);
        for (int P = I_NPL; P <= I_SPL; ++P)
          if (r_from == t->rgn4pl[P])
            for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k)
              VPL(var_pl[pole_rank], 1, k, P, v) = VAR(var[r], e[2], k, e[3], v);
      }
    }
  }
  {
    const rank_state *R = &t->rk[pole_rank];
    for (int i = 0; i < R->copy_p2r.n; ++i) {
      const int *e = R->copy_p2r.e + 4 * i;
      int r_from = LP2R(t, e[3], pole_rank + 1);
      if (r_from == t->rgn4pl[I_NPL] || r_from == t->rgn4pl[I_SPL])
        for (int v = 1; v <= vmax; ++v) for (int k = 1; k <= kmax; ++k)
          VPL(var_pl[pole_rank], e[0], k, e[1], v) = VAR(var[pole_rank], e[2], k, e[3], v);
    }
  }
  orc_comm_data_transfer(t, var, var_pl, kmax, vmax);
}

/* single-process transfer used inside the limiter (nprocs must be 1) */
void orc_comm_single(const orc_topo *t, double *var, double *var_pl, int kmax, int vmax) {
  double *v1[1] = {var}, *p1[1] = {var_pl};
  orc_comm_data_transfer(t, v1, p1, kmax, vmax);
}

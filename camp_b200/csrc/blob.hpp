// Compact mechanism tables for the solve kernel.  The host packs them into one
// 16-byte aligned blob; every block copies the blob into the front of its
// shared memory with one bulk (TMA) copy, and all warps of the block read it
// from there.  Offsets are in bytes from the start of the blob, whose first
// kBlobHeader bytes hold the BlobOff itself.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace campb {

struct BlobOff {
  int bytes;        // whole blob
  int stage_bytes;  // prefix the level-scheduled mode stages (all but the one-lane LU)
  // counts
  int n, n_rxn, n_part, n_jac, n_lu, n_coef, n_funits, n_fsplit, n_fscratch;
  int n_plev, n_flev, n_blev;
  // reactions: variable reactants packed (nv<<30 | d2<<20 | d1<<10 | d0), partial base
  int rx_word, rx_vptr;
  // coefficient table (double)
  int coef;
  // f gather: entries (rxn | coef<<16 | prod<<31), units (species, begin, end,
  // slot) as 4 x uint16, lane pointers (33 x uint16), split species (species,
  // first slot, count) as 3 x uint16
  int fg_ent, fg_unit, fg_lane, fg_split;
  // J gather: w0 = part | coef<<16, w1 = independent species + 1 (0 = loss
  // entry); per slot: entry pointer, LU position, row; lane slot lists
  int jg_w0, jg_w1, jg_ptr, jg_mid, jg_lupos, jg_row, jg_lane, jg_slots;
  // LU: perm, diag (uint16); factorization by pivot level: scaled L entries
  // (fa_ptr uint16, fa = pos | pivot<<16), Schur updates grouped by target
  // with the reciprocal pivots taken in the same phase (fb); forward solve
  // (fw); backward solve updates with the pivots finalised in the same
  // phase (bw).  A grouped phase G has round pointers per level (uint16,
  // levels + 1; the *_lane fields), one record per lane and round (the
  // *_unit fields: uint32 target | count<<16, uint32 first pair |
  // (pivot+1)<<16, pivot 0 = none; a no-op record targets the spare slot
  // past the accumulator) and pairs (uint32 a | b<<16).
  int lu_perm, lu_diag, lu_src;
  int fa_ptr, fa;
  int fb_lane, fb_unit, fb_pair;
  int fw_lane, fw_unit, fw_pair;
  int bw_lane, bw_unit, bw_pair;
  // row-wise LU for the sequential (one-lane) mode: J slot -> LU position
  // (jg_lupos), diagonal positions, rowptr, col (uint16), update pointer per
  // L entry (uint32) and updates (src | dst<<16); staged only in that mode
  int lu_rowptr, lu_col, upd_ptr, upd;
  // dependent index -> state index (uint16); absolute tolerances (double)
  int dep_state, atol;
  // SIMPOL phase transfer: per instance a record of 8 x uint16 (gas and
  // aerosol dependent indices, dependent element count, first element, first
  // Jacobian partial), per dependent element its index (uint16) and factors
  // (1/density, 1/MW when in the instance's phase else 0, in-phase flag;
  // 3 x double).  Its 4 pseudo-rates per instance follow the terms' rates,
  // its 8 per-cell constants the terms' rate constants.
  int n_simpol, n_keff, n_rates, n_part_all;
  int si_rec, si_elem, si_ef;
  // aqueous equilibrium instances: record (uint16 x 12: dependent slots,
  // dependent reactant slots, first slot, first pseudo-rate, first partial,
  // keff slot, computed water | reactant and product counts, computed
  // activity coefficient, first and count of the computed participants),
  // per slot its dependent index (uint16) and 1e3 / MW (double); per
  // computed participant its computed index | reactant << 15 (uint16) and
  // 1e3 / MW (double)
  int n_aq, aq_rec, aq_sp, aq_sm, aq_cp, aq_cpm;
  int aq_sim;  // per slot MW / 1e3 (1 / aq_sm), double
  // J gather with unguarded products (SIMPOL): they lead each slot, and
  // jg_umid (uint16 per slot) is the slot's first loss entry
  int has_ug, jg_umid;
  // sub-models: computed species, parameter-Jacobian elements, keff slot of
  // PPM_TO_RH_; per computed species its program's first int and first
  // float (2 x uint32), the program ints (int32) and floats (double).  The
  // values sit after the pseudo-rates (f) or the partials (J), the
  // parameter partials and the virtual slots after the values.
  int n_cv, n_pj, sm_keff, sm_rec, sm_int, sm_flt;
  int sm_state;  // state index of each computed species (uint16)
  // virtual Jacobian slots: partial lists (uint16 pointers, n_virt + 1, and
  // uint16 partial indices); the chain by target slot: target (uint16),
  // entry pointers (uint16, n_chain + 1), entries (uint32: virtual slot |
  // parameter id << 16)
  int n_virt, jv_ptr, jv_part, n_chain, ch_tgt, ch_ptr, ch_ent;
};

constexpr int kBlobHeader = 512;

struct Tables;

// Builds the blob; false (with a message) if the mechanism exceeds the
// encodings (more than 3 variable reactants in a reaction, more than 1023
// dependent variables, or index spaces beyond 16 bits).
bool build_blob(const Tables& t, const std::vector<double>& atol_dep,
                std::vector<uint8_t>* blob, BlobOff* off, std::string* err);

}  // namespace campb

namespace campb {

// Tables of the lane-per-cell kernel (one cell per lane, all lanes of a warp
// read the same table entry at the same time).  Header first, then sections;
// offsets in bytes from the start of the blob.
struct LaneOff {
  int bytes;
  int n, n_rxn, n_lu, n_coef, n_part, n_jpos, n_upd;
  // reactions: variable reactants (nv<<30 | d2<<20 | d1<<10 | d0, uint32);
  // participants (variable reactant occurrences, then variable products) per
  // reaction: pointer (uint16) and entries (species | coef<<10 | product<<31)
  int rx_word, rx_pptr, rx_part;
  // Jacobian scatter: per reaction, for each variable reactant occurrence k
  // and each participant p, the LU position of d(p)/d(k) (uint16)
  int rx_jptr, jpos;
  int coef;  // double
  // row-wise LU in pivot order (uint16) and update lists (uint32)
  int lu_perm, lu_rowptr, lu_col, lu_diag, upd_ptr, upd;
  int dep_state;  // uint16
  int atol;       // double
};

bool build_lane_blob(const Tables& t, const std::vector<double>& atol_dep,
                     std::vector<uint8_t>* blob, LaneOff* off, std::string* err);

}  // namespace campb

namespace campb {

// Tables of the CTA-per-cell kernel (one thread block per cell), for
// mechanisms whose LU is too large for the warp-per-cell tables.  The block
// reads them from global memory through L1.  The LU is row-wise in pivot
// order with sorted columns; its trailing rows r0..n-1 form a dense block
// (every column r0..n-1 present), addressed without tables: entry (i, j) of
// that block sits at dpos[i - r0] + (j - r0).  The sparse head (pivots and
// rows before r0) is factored pivot by pivot from tabulated update targets
// and solved by row levels.  Offsets in bytes from the start of the blob.
struct BlockOff {
  int bytes;
  int n, n_rxn, n_part, n_jac, n_lu, n_coef;
  int r0;          // first row (pivot) of the trailing dense block
  int n_hf, n_hb;  // forward / backward row levels of the head rows
  // reactions: variable reactants (nv<<30 | d2<<20 | d1<<10 | d0, uint32)
  // and the first rate partial of each (uint32, n_rxn + 1)
  int rx_word, rx_vptr;
  int coef;  // double
  // f gather by species: pointers (uint32, n + 1), entries (uint32: term |
  // coef<<16 | guarded product<<31)
  int fg_ptr, fg_ent;
  // J gather by solver slot: pointers (uint32, n_jac + 1), first guarded
  // product (uint32), entries (uint32: partial | coef<<16), guard species + 1
  // (uint16), row species (uint16)
  int jg_ptr, jg_mid, jg_w0, jg_w1, jg_row;
  // per LU position: J slot + 1 (0 = none) | diagonal<<15 (uint16)
  int lu_src;
  // LU structure (uint16): pivot -> dependent index, row pointers, columns,
  // diagonal positions
  int lu_perm, lu_rowptr, lu_col, lu_diag;
  int dpos;  // per dense row: position of its column r0 (uint16)
  int ub;    // per head row: first position with a column >= r0 (uint16)
  // head pivots k < r0: L entries of column k in row order (pointers
  // uint32, r0 + 1; entries uint32: position | row << 16), the first of
  // them in a dense row (uint32 per pivot), and the tabulated updates
  // (pointers uint32, r0 + 1; records uint64: target | L position << 16 |
  // U position << 32): the head rows' L entries against every U entry of
  // row k, then the dense rows' against the U entries of row k in head
  // columns, row-major.  The dense rows' updates in dense columns are
  // addressed through the dense block.
  int lk_ptr, lk, lk_mid, tg_ptr, hrec;
  // head row levels (pointers uint16, levels + 1; rows uint16)
  int hf_ptr, hf_rows, hb_ptr, hb_rows;
  int dep_state;  // uint16
  int atol;       // double
  // the solve's tables, one uint16 section the block copies into shared
  // memory (stage: byte offset, sg_len: elements); element offsets inside:
  // row pointers (n + 1), diagonals (n), head rows' ub (r0), permutation
  // (n), head levels (forward pointers and rows, backward pointers and
  // rows), per row the first of its non-dense entries in ndcol (n + 1; the
  // head rows' entries, the dense rows' head-column entries) and their
  // columns, and the dense rows' bases (dpos - r0, m)
  int stage, sg_len;
  int sg_rowptr, sg_diag, sg_ub, sg_perm, sg_hf_ptr, sg_hf_rows, sg_hb_ptr, sg_hb_rows;
  int sg_ndoff, sg_ndcol, sg_dbase;
  // and the head pivots' pointers: lk_ptr (r0 + 1), lk_mid (r0), tg_ptr
  // (r0 + 1), as uint16
  int sg_hlk, sg_hmid, sg_htg;
};

// the largest trailing dense block the CTA kernel holds in registers
// (a 16 x 16 thread grid, 7 x 7 entries per thread)
constexpr int kBlockMaxDense = 112;

bool build_block_blob(const Tables& t, const std::vector<double>& atol_dep,
                      std::vector<uint8_t>* blob, BlockOff* off, std::string* err);

}  // namespace campb

/*
 * Test-infrastructure harness: exposes the reference's OWN counting kernels
 * (static inline functions of src/command_ani.h) behind plain C entry points so
 * the oracle restatement and the CUDA path can be compared with the reference
 * itself on arbitrary inputs.  Built only into oracle/_ref/ (never shipped).
 *
 *   refh_count_block -> count_ctx_obj_frm_comb_sketch_section_with_unique
 *                       (src/command_ani.h:463-624), matrix mode (no filtering)
 *   refh_count_lower -> count_ctx_obj_frm_comb_sketch_section_lower
 *                       (src/command_ani.h:635-721)
 *   refh_count_detail-> the same with fmt==0: ctxcut / afcut / float naive-ANI
 *                       pre-filter and top-N ranking (src/command_ani.h:577-621)
 *   refh_pair_features -> get_ani_features_ctx_min_over_conflicts_both_filtered
 *                       (src/command_ani.h:303-346)
 */
#include "command_ani.h"

int ani_model_drfold;

static void set_bits(int obj_bits)
{
	Bitslen.obj = (uint8_t)obj_bits;
	Bitslen.ctx = (uint8_t)(64 - 20 > obj_bits ? 44 : 0);
	Bitslen.gid = 20;
}

static ani_opt_t base_opt(int threads, int ignoreconflict)
{
	ani_opt_t o;
	memset(&o, 0, sizeof(o));
	o.fmt = 1;
	o.p = threads > 0 ? threads : 1;
	o.ignoreconflict = ignoreconflict != 0;
	o.ntop = -1;
	o.ctxcut = 3;
	o.afcut = 0.5f;
	o.anicut = 0.95f;
	o.s = 1;
	o.e = 1;
	o.max_diff_obj_section = -1;
	return o;
}

int refh_count_block(const void *index12, size_t index_len, int nref,
					 const uint64_t *qkeys, const uint64_t *qoffs, int nq,
					 int obj_bits, int ignoreconflict, int want_unique, int threads,
					 uint32_t *ctx2, uint32_t *obj2, uint32_t *uctx2, uint32_t *uobj2)
{
	set_bits(obj_bits);
	ani_opt_t o = base_opt(threads, ignoreconflict);
	o.unique_ctx = want_unique != 0;
	count_ctx_obj_frm_comb_sketch_section_with_unique(
		(ctx_mut2_t *)ctx2, (obj_section_t *)obj2, (ctxgidobj_t *)index12, index_len, nref,
		NULL, NULL, nq, (uint64_t *)qkeys, (uint64_t *)qoffs, NULL, NULL, &o,
		want_unique ? (ctx_mut2_t *)uctx2 : NULL, want_unique ? (obj_section_t *)uobj2 : NULL, NULL);
	return 0;
}

int refh_count_lower(const void *index12, size_t index_len, int nref, int qry_gid_offset,
					 const uint64_t *qkeys, const uint64_t *qoffs, int nq,
					 int obj_bits, int ignoreconflict, int threads,
					 uint32_t *ctx2, uint32_t *obj2)
{
	set_bits(obj_bits);
	ani_opt_t o = base_opt(threads, ignoreconflict);
	count_ctx_obj_frm_comb_sketch_section_lower(
		(ctx_mut2_t *)ctx2, (obj_section_t *)obj2, (ctxgidobj_t *)index12, index_len, nref,
		qry_gid_offset, nq, (uint64_t *)qkeys, (uint64_t *)qoffs, &o);
	return 0;
}

int refh_count_detail(const void *index12, size_t index_len, int nref,
					  const uint64_t *qkeys, const uint64_t *qoffs, int nq,
					  int obj_bits, int ignoreconflict, int want_unique, int threads,
					  const uint32_t *ref_ctx_count, const uint32_t *qry_ctx_count,
					  int ctxcut, float afcut, float anicut, int ntop,
					  uint32_t *ctx2, uint32_t *obj2, uint32_t *uctx2, uint32_t *uobj2,
					  uint32_t *num_pass, uint32_t *ranked_ids)
{
	set_bits(obj_bits);
	ani_opt_t o = base_opt(threads, ignoreconflict);
	o.fmt = 0;
	o.unique_ctx = want_unique != 0;
	o.ctxcut = ctxcut;
	o.afcut = afcut;
	o.anicut = anicut;
	o.ntop = ntop;
	idani_t **rank = malloc((size_t)nq * sizeof(*rank));
	for (int i = 0; i < nq; i++)
		rank[i] = malloc((size_t)nref * sizeof(idani_t));
	count_ctx_obj_frm_comb_sketch_section_with_unique(
		(ctx_mut2_t *)ctx2, (obj_section_t *)obj2, (ctxgidobj_t *)index12, index_len, nref,
		ref_ctx_count, qry_ctx_count, nq, (uint64_t *)qkeys, (uint64_t *)qoffs, num_pass, rank, &o,
		want_unique ? (ctx_mut2_t *)uctx2 : NULL, want_unique ? (obj_section_t *)uobj2 : NULL, NULL);
	for (int i = 0; i < nq; i++) {
		for (uint32_t k = 0; k < num_pass[i]; k++)
			ranked_ids[(size_t)i * nref + k] = rank[i][k].id;
		free(rank[i]);
	}
	free(rank);
	return 0;
}

int refh_pair_features(const uint64_t *a, size_t n, const uint64_t *b, size_t m,
					   int obj_bits, int ignore_b_conflict, uint32_t out4[4])
{
	set_bits(obj_bits);
	ani_features_t f;
	get_ani_features_ctx_min_over_conflicts_both_filtered(a, n, b, m, ignore_b_conflict != 0, &f);
	out4[0] = f.XnY_ctx;
	out4[1] = f.N_diff_obj;
	out4[2] = f.N_diff_obj_section;
	out4[3] = f.N_mut2_ctx;
	return 0;
}

/* The reference's FP64 model functions (src/model_ani.h, src/model_refaf_hgb.h,
 * src/command_ani.h:200-232, src/command_matrix.c:26-33), for bit-exact tests of the
 * host epilogue.  f5 = {XnY, X_ctx, section, mut2, diff_obj} as ani_features_t. */
extern double get_mashD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY);
extern double get_aafD(uint32_t K, uint32_t X, uint32_t Y, uint32_t XnY);

void refh_models(const uint32_t *f5, int drfold, int obj_bits, double out[6])
{
	set_bits(obj_bits);
	ani_model_drfold = drfold;
	ani_features_t f;
	memcpy(&f, f5, sizeof f);
	ani_features_t t = f;
	out[0] = lm3ways_dist_from_features(&t);
	t = f;
	out[1] = lm3ways_af_ANIb_from_features(&t);
	t = f;
	out[2] = get_naive_dist(&t);
	t = f;
	out[3] = get_p_dist(&t);
	out[4] = get_mashD(Bitslen.ctx / 2, f.X_ctx, f.XnY_ctx + 7, f.XnY_ctx);
	out[5] = get_aafD(Bitslen.ctx / 2, f.X_ctx, f.XnY_ctx + 7, f.XnY_ctx);
}

double refh_hgb(double raw_ani, double ref_af, unsigned xny, unsigned dobj, unsigned sect, unsigned mut2, int drfold)
{
	ani_model_drfold = drfold;
	return refaf_hgb_predict_ani(raw_ani, ref_af, xny, dobj, sect, mut2);
}

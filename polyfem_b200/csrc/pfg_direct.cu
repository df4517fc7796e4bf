// Sparse direct solve on the device: a multifrontal Cholesky factorisation
// P A P^T = L L^T of a symmetric positive definite matrix in the assembler's CSC
// pattern, and the triangular solves.  PolyFEM's Newton step hands each assembled
// Hessian to a polysolve linear::Solver (analyzePattern, factorize, solve) inside
// the Newton solver of polysolve@47dc48d (external); the direct choices its call
// sites name are sparse LDL^T / Cholesky factorisations (Eigen::SimplicialLDLT,
// Cholmod, Pardiso: mesh/remesh/L2Projection.cpp:25-29, State.cpp:1562-1565).
// This is that family's algorithm laid out for the GPU:
//   analysis (host, once per pattern): columns with identical patterns (the dofs
//     of one node) are grouped; the group graph is ordered by nested dissection
//     with breadth-first level separators; the dissection tree is the assembly
//     tree: every separator (and every leaf part) is one front whose columns are
//     eliminated together, after its two halves.  Row structures, front sizes,
//     the scatter of A's entries into the fronts and the extend-add maps are
//     precomputed.
//   factorisation (device): fronts of equal height in the tree are processed by
//     the same launches, leaves first: A's lower entries are scattered into the
//     zeroed fronts, the children's update matrices are added in child order,
//     and each front is partially factorised in pairs of 32-column panels
//     (Cholesky of each diagonal block, triangular solve of the rows below, the
//     first panel's update of the second, then one rank-64 update of the trailing
//     lower triangle in 64 x 64 tiles); the trailing block is the update matrix
//     the parent adds.
//   solve (device): forward substitution leaves first (each front adds its
//     children's update vectors in child order), backward substitution from the
//     root, then the inverse permutation.
// Every sum is taken in a fixed order, so factor and solution are bitwise
// deterministic.  Fronts are dense lower triangles of m (m + 1) / 2 doubles
// (packed columns), all resident for the factor's lifetime.
#include "pfg_internal.h"
#include "pfgpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace pfg
{

namespace
{

constexpr int NB = 32;          // panel width of the triangular solves
constexpr int NBF = 64;         // panel width of the partial factorisation
constexpr int LEAF_DOFS = 96;   // dissection stops at parts of at most this many dofs
constexpr int TRSM_ROWS = 128;  // rows per CTA of the panel solve
constexpr int TILE = 64;        // trailing-update tile
constexpr int FWD_ROWS = 256;   // rows per CTA of the forward solve's panel update
constexpr int BWD_ROWS = 512;   // rows per CTA of the backward solve's panel sums

struct DevFront
{
	long long foff; // front in the front buffer (doubles): m (m + 1) / 2, packed lower columns
	long long woff; // m doubles of solve workspace
	long long roff; // rows of this front's update in the parent (relpos), m - k entries
	long long ioff; // permuted positions of the m - k rows below the front's columns
	int col0;       // first permuted column
	int k;          // columns eliminated in this front
	int m;          // k + rows below
	int child0;     // children in child_list[child0 .. child0 + nchild)
	int nchild;
	int pad;
};

// Fronts are stored as packed lower columns: column j of an order-m front holds
// rows j .. m-1, and entry (i, j), i >= j, sits at pk(m, j) + i.
__host__ __device__ __forceinline__ long long pk(int m, int j) { return (long long)j * m - (long long)j * (j + 1) / 2; }

struct Panel
{
	int lvl, j0, rows_grid, tiles_grid;
	int fwd_grid, bwd_grid; // CTAs per front of the solve's panel steps
};

} // namespace

struct DirectFactor
{
	int n = 0;
	long long nnz = 0;
	int ns = 0;
	std::vector<int> perm;             // permuted position -> dof
	std::vector<DevFront> fr;          // fronts in postorder
	std::vector<int> lvl_start;        // fronts of height h: lvl_list[lvl_start[h] .. lvl_start[h+1])
	std::vector<int> lvl_list;
	std::vector<long long> lvl_fbeg;   // front doubles of each level [lvl_fbeg[h], lvl_fbeg[h+1])
	std::vector<long long> lvl_abeg;   // A-map entries of each level
	std::vector<int> lvl_maxchild, lvl_maxrc, lvl_maxk;
	int max_bwd_part = 0; // doubles of backward partial sums for one panel step
	std::vector<Panel> panels;         // solve panels (NB columns) in order
	std::vector<Panel> fpanels;        // factorisation panels (NBF columns) in order
	long long front_doubles = 0, work_doubles = 0, amap_n = 0;
	// host maps between the analysis and the upload
	std::vector<int> h_child, h_relpos, h_rows, h_amap_src;
	std::vector<long long> h_amap_dst;
	// device
	DevFront *d_fr = nullptr;
	int *d_lvl_list = nullptr, *d_child = nullptr, *d_relpos = nullptr, *d_rows = nullptr, *d_perm = nullptr;
	int *d_amap_src = nullptr;
	long long *d_amap_dst = nullptr;
	double *d_front = nullptr, *d_work = nullptr, *d_vec = nullptr; // d_vec: 2 n (permuted rhs, solution)
	double *d_io = nullptr;                                          // n: b and x of a host-memory solve
	double *d_part = nullptr;                                        // backward panel partial sums
	int *d_err = nullptr;
	bool factorized = false;
};

// ------------------------------------------------------------------ analysis

namespace
{

struct NdBuilder
{
	// group graph
	int nv = 0;
	std::vector<int> off, adj, wt;
	// dissection tree (created in postorder: every node after its descendants)
	std::vector<std::vector<int>> cols;     // groups of each node
	std::vector<std::vector<int>> children;
	std::vector<int> mark, vis, lev;
	int label = 0, stamp = 0;

	int make_node(std::vector<int> g, std::vector<int> ch)
	{
		std::sort(g.begin(), g.end());
		cols.push_back(std::move(g));
		children.push_back(std::move(ch));
		return (int)cols.size() - 1;
	}

	// breadth-first levels from root over vertices marked `lab`; returns the visit
	// order and fills level starts; vis[] = stamp for visited, lev[] = level
	void bfs(int root, int lab, std::vector<int> &order, std::vector<int> &ls)
	{
		++stamp;
		order.clear();
		ls.clear();
		order.push_back(root);
		vis[root] = stamp;
		lev[root] = 0;
		ls.push_back(0);
		size_t head = 0;
		int cur = 0;
		while (head < order.size())
		{
			const int v = order[head];
			if (lev[v] != cur)
			{
				cur = lev[v];
				ls.push_back((int)head);
			}
			++head;
			for (int t = off[v]; t < off[v + 1]; ++t)
			{
				const int u = adj[t];
				if (mark[u] == lab && vis[u] != stamp)
				{
					vis[u] = stamp;
					lev[u] = lev[v] + 1;
					order.push_back(u);
				}
			}
		}
		ls.push_back((int)order.size());
	}

	int degree_in(int v, int lab) const
	{
		int d = 0;
		for (int t = off[v]; t < off[v + 1]; ++t) d += mark[adj[t]] == lab;
		return d;
	}

	// nested dissection of the vertex set S; returns the roots of its subtrees
	std::vector<int> build(std::vector<int> S)
	{
		std::vector<int> roots;
		if (S.empty()) return roots;
		const int lab = ++label;
		for (int v : S) mark[v] = lab;
		std::vector<int> order, ls;
		bfs(S[0], lab, order, ls);
		if (order.size() < S.size())
		{
			// disconnected: every component is its own subtree
			std::vector<std::vector<int>> comps;
			comps.push_back(order);
			for (int v : order) mark[v] = -1;
			for (int v : S)
				if (mark[v] == lab)
				{
					bfs(v, lab, order, ls);
					comps.push_back(order);
					for (int u : order) mark[u] = -1;
				}
			for (auto &c : comps)
			{
				std::vector<int> r = build(std::move(c));
				roots.insert(roots.end(), r.begin(), r.end());
			}
			return roots;
		}
		long long w = 0;
		for (int v : S) w += wt[v];
		if (w <= LEAF_DOFS)
		{
			roots.push_back(make_node(std::move(S), {}));
			return roots;
		}
		// pseudo-peripheral root: restart from a minimum-degree vertex of the last
		// level while the eccentricity grows
		int r = S[0], h = (int)ls.size() - 1;
		for (int it = 0; it < 4; ++it)
		{
			int best = -1, bd = 1 << 30;
			for (int q = ls[h - 1]; q < ls[h]; ++q)
			{
				const int d = degree_in(order[q], lab);
				if (d < bd) bd = d, best = order[q];
			}
			std::vector<int> o2, l2;
			bfs(best, lab, o2, l2);
			const int h2 = (int)l2.size() - 1;
			if (h2 <= h)
			{
				bfs(r, lab, order, ls); // restore r's levels
				break;
			}
			r = best;
			h = h2;
			order.swap(o2);
			ls.swap(l2);
		}
		if (h < 3)
		{
			roots.push_back(make_node(std::move(S), {}));
			return roots;
		}
		// separator level: the first level where the weight before it reaches half
		long long acc = 0;
		int mid = 1;
		for (int q = 0; q < h; ++q)
		{
			long long lw = 0;
			for (int t = ls[q]; t < ls[q + 1]; ++t) lw += wt[order[t]];
			if (acc + lw > w / 2)
			{
				mid = q;
				break;
			}
			acc += lw;
		}
		mid = std::min(std::max(mid, 1), h - 2);
		std::vector<int> A, B, Sep;
		for (int q = 0; q < h; ++q)
			for (int t = ls[q]; t < ls[q + 1]; ++t)
			{
				const int v = order[t];
				if (q < mid) A.push_back(v);
				else if (q > mid) B.push_back(v);
				else
				{
					// a level-mid vertex with no neighbour beyond the separator joins A
					bool beyond = false;
					for (int e = off[v]; e < off[v + 1] && !beyond; ++e)
					{
						const int u = adj[e];
						beyond = mark[u] == lab && vis[u] == stamp && lev[u] == mid + 1;
					}
					(beyond ? Sep : A).push_back(v);
				}
			}
		std::vector<int> ch = build(std::move(A));
		std::vector<int> cb = build(std::move(B));
		ch.insert(ch.end(), cb.begin(), cb.end());
		if (Sep.empty())
		{
			roots = ch;
			return roots;
		}
		roots.push_back(make_node(std::move(Sep), std::move(ch)));
		return roots;
	}
};

template <class T>
static cudaError_t upload(T **d, const std::vector<T> &h)
{
	*d = nullptr;
	const size_t bytes = sizeof(T) * std::max<size_t>(h.size(), 1);
	cudaError_t e = cudaMalloc(reinterpret_cast<void **>(d), bytes);
	if (e != cudaSuccess) return e;
	if (!h.empty()) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
	return e;
}

} // namespace

void direct_destroy(DirectFactor *f)
{
	if (!f) return;
	void *ptrs[] = {f->d_fr,       f->d_lvl_list, f->d_child, f->d_relpos, f->d_rows, f->d_perm, f->d_amap_src,
					f->d_amap_dst, f->d_front,    f->d_work,  f->d_vec,    f->d_io,   f->d_err, f->d_part};
	for (void *p : ptrs)
		if (p) cudaFree(p); // a host-only analysis never touches the runtime
	delete f;
}

int direct_n(const DirectFactor *f) { return f ? f->n : 0; }
long long direct_nnz(const DirectFactor *f) { return f ? f->nnz : 0; }
long long direct_front_bytes(const DirectFactor *f) { return f ? f->front_doubles * 8 : 0; }
int direct_fronts(const DirectFactor *f) { return f ? f->ns : 0; }
bool direct_factorized(const DirectFactor *f) { return f && f->factorized; }
double *direct_io(DirectFactor *f) { return f ? f->d_io : nullptr; }

// Host analysis of a pattern (full symmetric CSC, sorted rows, n > 0 columns):
// ordering, fronts and every index map, each checked against the front it
// addresses before anything reaches the device.  0 ok, else a PFG error code
// with msg; *out owns the host arrays (and the maps until direct_upload).
int direct_symbolic(int n, const int *outer, const int *inner, DirectFactor **out, std::string &msg)
{
	*out = nullptr;
	auto *f = new DirectFactor();
	f->n = n;
	f->nnz = n > 0 ? outer[n] : 0;
	// 1. groups of consecutive columns with identical patterns
	std::vector<int> gof(n), gfirst;
	for (int j = 0; j < n; ++j)
	{
		bool same = false;
		if (j > 0)
		{
			const int a0 = outer[j - 1], a1 = outer[j], b0 = outer[j], b1 = outer[j + 1];
			same = (a1 - a0) == (b1 - b0) && std::equal(inner + a0, inner + a1, inner + b0);
		}
		if (same) gof[j] = gof[j - 1];
		else
		{
			gof[j] = (int)gfirst.size();
			gfirst.push_back(j);
		}
	}
	const int ng = (int)gfirst.size();
	gfirst.push_back(n);
	NdBuilder nd;
	nd.nv = ng;
	nd.off.assign(ng + 1, 0);
	nd.wt.assign(ng, 0);
	for (int g = 0; g < ng; ++g)
	{
		nd.wt[g] = gfirst[g + 1] - gfirst[g];
		const int j = gfirst[g];
		int last = -1;
		for (int t = outer[j]; t < outer[j + 1]; ++t)
		{
			const int h = gof[inner[t]];
			if (h != g && h != last) nd.adj.push_back(h);
			last = h;
		}
		nd.off[g + 1] = (int)nd.adj.size();
	}
	nd.mark.assign(ng, 0);
	nd.vis.assign(ng, 0);
	nd.lev.assign(ng, 0);
	std::vector<int> all(ng);
	std::iota(all.begin(), all.end(), 0);
	nd.build(std::move(all));
	const int ns = (int)nd.cols.size();
	f->ns = ns;
	// 2. permutation: columns in node (postorder) order
	std::vector<int> parent(ns, -1), col0(ns), kc(ns);
	for (int s = 0; s < ns; ++s)
		for (int c : nd.children[s]) parent[c] = s;
	f->perm.resize(n);
	std::vector<int> iperm(n);
	int pos = 0;
	for (int s = 0; s < ns; ++s)
	{
		col0[s] = pos;
		for (int g : nd.cols[s])
			for (int j = gfirst[g]; j < gfirst[g + 1]; ++j)
			{
				f->perm[pos] = j;
				iperm[j] = pos++;
			}
		kc[s] = pos - col0[s];
	}
	if (pos != n)
	{
		msg = "direct solver analysis lost columns";
		direct_destroy(f);
		return PFG_ERR_STATE;
	}
	// 3. row structures below each front's columns
	std::vector<std::vector<int>> rows(ns);
	for (int s = 0; s < ns; ++s)
	{
		const int last = col0[s] + kc[s] - 1;
		std::vector<int> R;
		for (int q = col0[s]; q <= last; ++q)
		{
			const int j = f->perm[q];
			for (int t = outer[j]; t < outer[j + 1]; ++t)
			{
				const int p = iperm[inner[t]];
				if (p > last) R.push_back(p);
			}
		}
		for (int c : nd.children[s])
			for (int p : rows[c])
				if (p > last) R.push_back(p);
		std::sort(R.begin(), R.end());
		R.erase(std::unique(R.begin(), R.end()), R.end());
		rows[s] = std::move(R);
	}
	// 4. heights and levels
	std::vector<int> height(ns, 0);
	int maxh = 0;
	for (int s = 0; s < ns; ++s)
	{
		for (int c : nd.children[s]) height[s] = std::max(height[s], height[c] + 1);
		maxh = std::max(maxh, height[s]);
	}
	const int nl = ns > 0 ? maxh + 1 : 0;
	f->lvl_start.assign(nl + 1, 0);
	for (int s = 0; s < ns; ++s) f->lvl_start[height[s] + 1]++;
	for (int h = 0; h < nl; ++h) f->lvl_start[h + 1] += f->lvl_start[h];
	f->lvl_list.resize(ns);
	{
		std::vector<int> fill(f->lvl_start.begin(), f->lvl_start.end() - 1);
		for (int s = 0; s < ns; ++s) f->lvl_list[fill[height[s]]++] = s;
	}
	// 5. fronts (allocated level by level), maps
	f->fr.resize(ns);
	std::vector<int> child_list, relpos, rowsflat;
	f->lvl_fbeg.assign(nl + 1, 0);
	f->lvl_abeg.assign(nl + 1, 0);
	f->lvl_maxchild.assign(nl, 0);
	f->lvl_maxrc.assign(nl, 0);
	long long fo = 0, wo = 0;
	std::vector<int> amap_src;
	std::vector<long long> amap_dst;
	// local index of permuted position p in front s's list, -1 if absent
	auto local = [&](int s, int p) -> int {
		const int last = col0[s] + kc[s] - 1;
		if (p <= last) return p >= col0[s] ? p - col0[s] : -1;
		const auto &R = rows[s];
		const auto it = std::lower_bound(R.begin(), R.end(), p);
		return it != R.end() && *it == p ? kc[s] + (int)(it - R.begin()) : -1;
	};
	bool broken = false;
	for (int s = 0; s < ns; ++s)
	{
		DevFront &d = f->fr[s];
		d.col0 = col0[s];
		d.k = kc[s];
		d.m = kc[s] + (int)rows[s].size();
		d.child0 = (int)child_list.size();
		d.nchild = (int)nd.children[s].size();
		d.pad = 0;
		for (int c : nd.children[s]) child_list.push_back(c);
		d.ioff = (long long)rowsflat.size();
		rowsflat.insert(rowsflat.end(), rows[s].begin(), rows[s].end());
		d.woff = wo;
		wo += d.m;
	}
	for (int s = 0; s < ns; ++s)
	{
		DevFront &d = f->fr[s];
		d.roff = (long long)relpos.size();
		if (parent[s] >= 0)
		{
			int prev = -1;
			for (int p : rows[s])
			{
				const int l = local(parent[s], p);
				broken |= l <= prev; // present in the parent, increasing
				relpos.push_back(l);
				prev = l;
			}
		}
		else broken |= !rows[s].empty();
	}
	for (int h = 0; h < nl; ++h)
	{
		f->lvl_fbeg[h] = fo;
		f->lvl_abeg[h] = (long long)amap_src.size();
		for (int t = f->lvl_start[h]; t < f->lvl_start[h + 1]; ++t)
		{
			const int s = f->lvl_list[t];
			DevFront &d = f->fr[s];
			d.foff = fo;
			fo += (long long)d.m * (d.m + 1) / 2;
			f->lvl_maxchild[h] = std::max(f->lvl_maxchild[h], d.nchild);
			for (int c : nd.children[s]) f->lvl_maxrc[h] = std::max(f->lvl_maxrc[h], f->fr[c].m - f->fr[c].k);
			for (int q = d.col0; q < d.col0 + d.k; ++q)
			{
				const int j = f->perm[q], cl = q - d.col0;
				for (int t2 = outer[j]; t2 < outer[j + 1]; ++t2)
				{
					const int p = iperm[inner[t2]];
					if (p < q) continue; // the upper entry of the pair
					const int lr = local(s, p);
					broken |= lr < cl || lr >= d.m; // lower triangle of this front
					amap_src.push_back(t2);
					amap_dst.push_back(d.foff + pk(d.m, cl) + lr);
				}
			}
		}
	}
	f->lvl_fbeg[nl] = fo;
	f->lvl_abeg[nl] = (long long)amap_src.size();
	f->front_doubles = fo;
	f->work_doubles = wo;
	f->amap_n = (long long)amap_src.size();
	// 6. panel launches of the factorisation
	for (int h = 0; h < nl; ++h)
	{
		int maxk = 0;
		for (int t = f->lvl_start[h]; t < f->lvl_start[h + 1]; ++t) maxk = std::max(maxk, f->fr[f->lvl_list[t]].k);
		f->lvl_maxk.push_back(maxk);
		for (int j0 = 0; j0 < maxk; j0 += NBF)
		{
			// rows_grid: panel A's rows below; fwd_grid: rows of A's update of B (0 when
			// no front has a panel B); bwd_grid: panel B's rows below; tiles_grid: the
			// rank-64 trailing update
			long long ra = 0, ru = 0, rb = 0, tg = 0;
			for (int t = f->lvl_start[h]; t < f->lvl_start[h + 1]; ++t)
			{
				const DevFront &d = f->fr[f->lvl_list[t]];
				if (d.k <= j0) continue;
				const int na = std::min(NB, d.k - j0);
				ra = std::max(ra, ((long long)d.m - j0 - na + TRSM_ROWS - 1) / TRSM_ROWS);
				if (d.k > j0 + NB)
				{
					const int nbb = std::min(NB, d.k - j0 - NB);
					ru = std::max(ru, ((long long)d.m - j0 - NB + TRSM_ROWS - 1) / TRSM_ROWS);
					rb = std::max(rb, ((long long)d.m - j0 - NB - nbb + TRSM_ROWS - 1) / TRSM_ROWS);
				}
				const int nb = std::min(NBF, d.k - j0);
				const long long below = d.m - j0 - nb;
				const long long nt = (below + TILE - 1) / TILE;
				tg = std::max(tg, nt * (nt + 1) / 2);
			}
			if (tg > 0x7fffffffLL)
			{
				msg = "direct solver front too large";
				direct_destroy(f);
				return PFG_ERR_UNSUPPORTED;
			}
			f->fpanels.push_back({h, j0, (int)ra, (int)tg, (int)ru, (int)rb});
		}
		for (int j0 = 0; j0 < maxk; j0 += NB)
		{
			long long rg = 0, tg = 0, fg = 0, bg = 1;
			for (int t = f->lvl_start[h]; t < f->lvl_start[h + 1]; ++t)
			{
				const DevFront &d = f->fr[f->lvl_list[t]];
				if (d.k <= j0) continue;
				const int nb = std::min(NB, d.k - j0);
				const long long below = d.m - j0 - nb;
				rg = std::max(rg, (below + TRSM_ROWS - 1) / TRSM_ROWS);
				const long long nt = (below + TILE - 1) / TILE;
				tg = std::max(tg, nt * (nt + 1) / 2);
				fg = std::max(fg, (below + FWD_ROWS - 1) / FWD_ROWS);
				bg = std::max(bg, ((long long)d.k - j0 - nb + BWD_ROWS - 1) / BWD_ROWS);
			}
			if (tg > 0x7fffffffLL)
			{
				msg = "direct solver front too large";
				direct_destroy(f);
				return PFG_ERR_UNSUPPORTED;
			}
			f->panels.push_back({h, j0, (int)rg, (int)tg, (int)fg, (int)bg});
			const long long nfl = f->lvl_start[h + 1] - f->lvl_start[h];
			f->max_bwd_part = (int)std::max<long long>(f->max_bwd_part, nfl * bg * NB);
		}
	}
	for (int h = 0; h < nl; ++h)
		if (f->lvl_start[h + 1] - f->lvl_start[h] > 65535)
		{
			msg = "direct solver: more than 65535 fronts of one height";
			direct_destroy(f);
			return PFG_ERR_UNSUPPORTED;
		}
	for (int s2 = 0; s2 < ns && !broken; ++s2)
	{
		const DevFront &d = f->fr[s2];
		broken |= d.k < 1 || d.m < d.k || d.foff < 0 || d.foff + (long long)d.m * (d.m + 1) / 2 > fo;
		const int last = d.col0 + d.k - 1;
		for (int q = 0; q < d.m - d.k && !broken; ++q)
		{
			const int p = rowsflat[d.ioff + q];
			broken |= p <= last || p >= n || (q > 0 && p <= rowsflat[d.ioff + q - 1]);
		}
	}
	if (broken)
	{
		msg = "direct solver analysis produced an inconsistent front structure";
		direct_destroy(f);
		return PFG_ERR_STATE;
	}
	f->h_child = std::move(child_list);
	f->h_relpos = std::move(relpos);
	f->h_rows = std::move(rowsflat);
	f->h_amap_src = std::move(amap_src);
	f->h_amap_dst = std::move(amap_dst);
	*out = f;
	return PFG_OK;
}

// the analysed maps to the device (the host copies are released); 0 ok, else a
// PFG error code with msg (f is left for direct_destroy)
int direct_upload(DirectFactor *f, std::string &msg)
{
	const int n = f->n;
	const long long fo = f->front_doubles, wo = f->work_doubles;
	// the fronts must fit beside what is already allocated
	size_t fre = 0, tot = 0;
	cudaError_t e = cudaMemGetInfo(&fre, &tot);
	if (e != cudaSuccess)
	{
		msg = cudaGetErrorString(e);
		return PFG_ERR_CUDA;
	}
	const double need = 8.0 * (double)fo + 8.0 * (double)wo + 12.0 * (double)f->amap_n + 24.0 * n + 8.0 * f->max_bwd_part;
	if (need > 0.85 * (double)fre)
	{
		msg = "direct solver needs " + std::to_string((long long)(need / 1e6)) + " MB of device memory for its fronts, " +
			  std::to_string((long long)(fre / 1000000)) + " MB free";
		return PFG_ERR_OOM;
	}
	if ((e = upload(&f->d_fr, f->fr)) != cudaSuccess || (e = upload(&f->d_lvl_list, f->lvl_list)) != cudaSuccess ||
		(e = upload(&f->d_child, f->h_child)) != cudaSuccess || (e = upload(&f->d_relpos, f->h_relpos)) != cudaSuccess ||
		(e = upload(&f->d_rows, f->h_rows)) != cudaSuccess || (e = upload(&f->d_perm, f->perm)) != cudaSuccess ||
		(e = upload(&f->d_amap_src, f->h_amap_src)) != cudaSuccess ||
		(e = upload(&f->d_amap_dst, f->h_amap_dst)) != cudaSuccess ||
		(e = cudaMalloc(&f->d_front, 8 * std::max<long long>(fo, 1))) != cudaSuccess ||
		(e = cudaMalloc(&f->d_work, 8 * std::max<long long>(wo, 1))) != cudaSuccess ||
		(e = cudaMalloc(&f->d_vec, 16 * (size_t)std::max(n, 1))) != cudaSuccess ||
		(e = cudaMalloc(&f->d_io, 8 * (size_t)std::max(n, 1))) != cudaSuccess ||
		(e = cudaMalloc(&f->d_part, 8 * (size_t)std::max(f->max_bwd_part, 1))) != cudaSuccess ||
		(e = cudaMalloc(&f->d_err, sizeof(int))) != cudaSuccess)
	{
		msg = cudaGetErrorString(e);
		return e == cudaErrorMemoryAllocation ? PFG_ERR_OOM : PFG_ERR_CUDA;
	}
	f->h_child = {};
	f->h_relpos = {};
	f->h_rows = {};
	f->h_amap_src = {};
	f->h_amap_dst = {};
	return PFG_OK;
}

void direct_stats(const DirectFactor *f, long long *st)
{
	// [n, fronts, levels, front doubles, nnz of L (columns of the fronts), largest
	// front, flops of the factorisation: column j of a front of order m updates the
	// (m-j-1)(m-j)/2 entries of its trailing lower triangle, one multiply-add each]
	long long nnzl = 0, mx = 0;
	double fl = 0.0;
	auto s2 = [](double t) { return t * (t + 1.0) * (2.0 * t + 1.0) / 6.0; }; // sum of squares 1..t
	auto s1 = [](double t) { return t * (t + 1.0) / 2.0; };
	for (const DevFront &d : f->fr)
	{
		nnzl += (long long)d.k * (d.k + 1) / 2 + (long long)d.k * (d.m - d.k);
		mx = std::max<long long>(mx, d.m);
		// sum over t = m-k .. m-1 of t (t + 1)
		const double hi = d.m - 1.0, lo = d.m - d.k - 1.0;
		fl += (s2(hi) - s2(lo)) + (s1(hi) - s1(lo));
	}
	st[6] = (long long)fl;
	st[0] = f->n;
	st[1] = f->ns;
	st[2] = (long long)f->lvl_start.size() - 1;
	st[3] = f->front_doubles;
	st[4] = nnzl;
	st[5] = mx;
}

// ------------------------------------------------------------------ kernels

namespace
{

__global__ void k_dir_assemble(long long n, const int *__restrict__ src, const long long *__restrict__ dst,
							   const double *__restrict__ vals, double *__restrict__ F)
{
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t < n) F[dst[t]] = vals[src[t]];
}

// child ci of every front of the level: F_s[relpos a, relpos b] += U_c[a, b] (a >= b);
// warp w of CTA x takes column b = 8 x + w of the child's update
__global__ void __launch_bounds__(256) k_dir_extend_add(const DevFront *__restrict__ fr, const int *__restrict__ list,
														const int *__restrict__ child, const int *__restrict__ relpos,
														double *__restrict__ F, int ci)
{
	const DevFront f = fr[list[blockIdx.y]];
	if (ci >= f.nchild) return;
	const DevFront c = fr[child[f.child0 + ci]];
	const int rc = c.m - c.k;
	const int b = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
	if (b >= rc) return;
	const int *rp = relpos + c.roff;
	const double *U = F + c.foff + pk(c.m, c.k + b) + c.k; // U[a] = entry (k + a, k + b), a >= b
	double *P = F + f.foff + pk(f.m, rp[b]);
	for (int a = b + lane; a < rc; a += 32) P[rp[a]] += U[a];
}

// Cholesky of the diagonal block of panel j0 (one warp per front): lane i holds row
// i of the block in registers; column c's entries reach the other lanes by shuffle
__global__ void __launch_bounds__(32) k_dir_potrf(const DevFront *__restrict__ fr, const int *__restrict__ list,
												  double *__restrict__ F, int j0, int *__restrict__ err)
{
	constexpr unsigned FULL = 0xffffffffu;
	const DevFront f = fr[list[blockIdx.x]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0), lane = threadIdx.x;
	double *Fb = F + f.foff;
	const bool row = lane < nb;
	double v[NB];
	{
		long long cb = pk(f.m, j0) + j0 + lane; // entry (j0 + lane, j0 + c)
#pragma unroll
		for (int c = 0; c < NB; ++c)
		{
			v[c] = row && c <= lane && c < nb ? Fb[cb] : 0.0;
			cb += f.m - (j0 + c) - 1;
		}
	}
	bool bad = false;
#pragma unroll
	for (int c = 0; c < NB; ++c)
	{
		if (c >= nb) break;
		double d = __shfl_sync(FULL, v[c], c);
		if (!(d > 0.0) || !(d <= 1.7976931348623157e308))
		{
			bad = true;
			d = 1.0;
		}
		d = sqrt(d);
		const double lc = lane == c ? d : (lane > c ? v[c] / d : 0.0); // L[lane][c]
		if (lane >= c) v[c] = lc;
#pragma unroll
		for (int l = c + 1; l < NB; ++l)
		{
			const double llc = __shfl_sync(FULL, lc, l); // L[l][c]
			if (lane >= l && l < nb) v[l] = fma(-lc, llc, v[l]);
		}
	}
	if (bad && lane == 0) atomicExch(err, 1);
	{
		long long cb = pk(f.m, j0) + j0 + lane;
#pragma unroll
		for (int c = 0; c < NB; ++c)
		{
			if (row && c <= lane && c < nb) Fb[cb] = v[c];
			cb += f.m - (j0 + c) - 1;
		}
	}
}

// rows below the panel: X L_d^T = B, one row per thread
__global__ void __launch_bounds__(TRSM_ROWS) k_dir_trsm(const DevFront *__restrict__ fr, const int *__restrict__ list,
														double *__restrict__ F, int j0)
{
	const DevFront f = fr[list[blockIdx.y]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0);
	__shared__ double D[NB][NB + 1];
	double *Fb = F + f.foff;
	for (int t = threadIdx.x; t < nb * nb; t += TRSM_ROWS)
	{
		const int r = t % nb, c = t / nb;
		if (r >= c) D[r][c] = Fb[(size_t)(j0 + r) + pk(f.m, j0 + c)];
	}
	__syncthreads();
	const long long i = (long long)j0 + nb + (long long)blockIdx.x * TRSM_ROWS + threadIdx.x;
	if (i >= f.m) return;
	double x[NB];
	const long long c0 = pk(f.m, j0) + i; // entry (i, j0); column j0 + l + 1 starts m - (j0 + l) - 1 later
	{
		long long cb = c0;
#pragma unroll
		for (int l = 0; l < NB; ++l)
		{
			if (l < nb) x[l] = Fb[cb];
			cb += f.m - (j0 + l) - 1;
		}
	}
#pragma unroll
	for (int l = 0; l < NB; ++l)
		if (l < nb)
		{
			double s = x[l];
#pragma unroll
			for (int t = 0; t < l; ++t) s = fma(-x[t], D[l][t], s);
			x[l] = s / D[l][l];
		}
	{
		long long cb = c0;
#pragma unroll
		for (int l = 0; l < NB; ++l)
		{
			if (l < nb) Fb[cb] = x[l];
			cb += f.m - (j0 + l) - 1;
		}
	}
}

// The factorisation runs in pairs of 32-column panels A = [j0, j0+32) and
// B = [j0+32, j0+64): A is factorised (k_dir_potrf, k_dir_trsm), its update is
// applied to B's columns alone (k_dir_panel_update), B is factorised, and one
// rank-64 update of the trailing lower triangle by both panels follows
// (k_dir_syrk64), so the trailing matrix is read and written once per 64 columns.
// k_dir_panel_update: F[i][j0+32+c] -= sum_l F[i][j0+l] F[j0+32+c][j0+l] for the
// rows i >= j0+32+c, a thread per row, A's rows of B's columns in shared memory.
__global__ void __launch_bounds__(TRSM_ROWS) k_dir_panel_update(const DevFront *__restrict__ fr,
																const int *__restrict__ list, double *__restrict__ F,
																int j0)
{
	const DevFront f = fr[list[blockIdx.y]];
	const int jb = j0 + NB;
	if (jb >= f.k) return;
	const int nc = min(NB, f.k - jb);
	__shared__ double M[NB][NB + 1]; // M[c][l] = F[jb + c][j0 + l]
	__shared__ long long cofs[NB];   // pk of columns j0 + l
	double *Fb = F + f.foff;
	if (threadIdx.x < NB) cofs[threadIdx.x] = pk(f.m, j0 + threadIdx.x);
	__syncthreads();
	for (int t = threadIdx.x; t < NB * NB; t += TRSM_ROWS)
	{
		const int c = t % NB, l = t / NB;
		M[c][l] = c < nc ? Fb[cofs[l] + jb + c] : 0.0;
	}
	__syncthreads();
	const long long i = (long long)jb + (long long)blockIdx.x * TRSM_ROWS + threadIdx.x;
	if (i >= f.m) return;
	double x[NB];
#pragma unroll
	for (int l = 0; l < NB; ++l) x[l] = Fb[cofs[l] + i];
	long long cb = pk(f.m, jb) + i; // entry (i, jb + c)
	for (int c = 0; c < nc; ++c)
	{
		if (i < jb + c) break; // upper part of B's block
		double a = 0.0;
#pragma unroll
		for (int l = 0; l < NB; ++l) a = fma(x[l], M[c][l], a);
		Fb[cb] -= a;
		cb += f.m - (jb + c) - 1;
	}
}

// trailing lower triangle -= P P^T for the pair's rows P below it (up to 64 columns),
// 64 x 64 tiles of the lower triangle, the two 64 x 64 row blocks of P in shared
// memory, 4 x 4 entries per thread
constexpr size_t SYRK64_SMEM = 2 * NBF * (TILE + 1) * sizeof(double);
__global__ void __launch_bounds__(256, 3) k_dir_syrk64(const DevFront *__restrict__ fr, const int *__restrict__ list,
													double *__restrict__ F, int j0)
{
	const DevFront f = fr[list[blockIdx.y]];
	if (j0 >= f.k) return;
	const int nb = min(NBF, f.k - j0);
	const int o = j0 + nb, t = f.m - o;
	if (t <= 0) return;
	const long long nt = (t + TILE - 1) / TILE;
	const long long tile = blockIdx.x;
	if (tile >= nt * (nt + 1) / 2) return;
	long long ti = (long long)((sqrt(8.0 * (double)tile + 1.0) - 1.0) * 0.5);
	while (ti * (ti + 1) / 2 > tile) --ti;
	while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
	const long long tj = tile - ti * (ti + 1) / 2;
	extern __shared__ __align__(16) double sy[];
	double(*Pi)[TILE + 1] = reinterpret_cast<double(*)[TILE + 1]>(sy);
	double(*Pj)[TILE + 1] = reinterpret_cast<double(*)[TILE + 1]>(sy + NBF * (TILE + 1));
	double *Fb = F + f.foff;
	__shared__ long long cofs[NBF]; // pk of columns j0 + l
	if (threadIdx.x < NBF) cofs[threadIdx.x] = pk(f.m, j0 + threadIdx.x);
	__syncthreads();
	// all of a thread's staging loads are issued before any is stored
	constexpr int SQ = NBF * TILE / 256;
	double vi[SQ], vj[SQ];
	const int r = threadIdx.x % TILE, l0 = threadIdx.x / TILE;
	const long long gi = ti * TILE + r, gj = tj * TILE + r;
#pragma unroll
	for (int q = 0; q < SQ; ++q)
	{
		const int l = l0 + q * (256 / TILE);
		const bool ok = l < nb;
		vi[q] = ok && gi < t ? Fb[cofs[l] + o + gi] : 0.0;
		vj[q] = ok && gj < t ? Fb[cofs[l] + o + gj] : 0.0;
	}
#pragma unroll
	for (int q = 0; q < SQ; ++q)
	{
		const int l = l0 + q * (256 / TILE);
		Pi[l][r] = vi[q];
		Pj[l][r] = vj[q];
	}
	__syncthreads();
	const int tr = (threadIdx.x % 16) * 4, tc = (threadIdx.x / 16) * 4;
	double acc[4][4] = {};
#pragma unroll 4
	for (int l = 0; l < NBF; ++l)
	{
		double a[4], b[4];
#pragma unroll
		for (int q = 0; q < 4; ++q)
		{
			a[q] = Pi[l][tr + q];
			b[q] = Pj[l][tc + q];
		}
#pragma unroll
		for (int p = 0; p < 4; ++p)
#pragma unroll
			for (int q = 0; q < 4; ++q) acc[p][q] = fma(a[p], b[q], acc[p][q]);
	}
	long long cb = pk(f.m, (int)(o + tj * TILE + tc)) + o + ti * TILE + tr; // entry (o + gr, o + gc) at p = q = 0
#pragma unroll
	for (int q = 0; q < 4; ++q)
	{
		const long long gc = tj * TILE + tc + q;
#pragma unroll
		for (int p = 0; p < 4; ++p)
		{
			const long long gr = ti * TILE + tr + p;
			if (gr < t && gc < t && gr >= gc) Fb[cb + p] -= acc[p][q];
		}
		cb += f.m - (o + gc) - 1;
	}
}

__global__ void k_dir_permute_in(int n, const int *__restrict__ perm, const double *__restrict__ b, double *__restrict__ bp)
{
	const int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q < n) bp[q] = b[perm[q]];
}

__global__ void k_dir_permute_out(int n, const int *__restrict__ perm, const double *__restrict__ xp, double *__restrict__ x)
{
	const int q = blockIdx.x * blockDim.x + threadIdx.x;
	if (q < n) x[perm[q]] = xp[q];
}

// Forward substitution, level by level from the leaves, in the factorisation's
// 32-column panels.  k_fwd_init: w = [b_cols; 0] plus the children's update
// vectors (one CTA per front, children in order); per panel, k_fwd_diag (one warp
// per front) solves the diagonal block in registers and k_fwd_rows updates the
// rows below it (a thread per row, several CTAs per front, coalesced columns of L).
__global__ void __launch_bounds__(256) k_fwd_init(const DevFront *__restrict__ fr, const int *__restrict__ list,
												  const int *__restrict__ child, const int *__restrict__ relpos,
												  const double *__restrict__ bp, double *__restrict__ W)
{
	const DevFront f = fr[list[blockIdx.x]];
	double *w = W + f.woff;
	for (int i = threadIdx.x; i < f.m; i += 256) w[i] = i < f.k ? bp[f.col0 + i] : 0.0;
	__syncthreads();
	for (int ci = 0; ci < f.nchild; ++ci)
	{
		const DevFront c = fr[child[f.child0 + ci]];
		const int rc = c.m - c.k;
		const int *rp = relpos + c.roff;
		const double *wc = W + c.woff + c.k;
		for (int i = threadIdx.x; i < rc; i += 256) w[rp[i]] += wc[i];
		__syncthreads();
	}
}

__global__ void __launch_bounds__(32) k_fwd_diag(const DevFront *__restrict__ fr, const int *__restrict__ list,
												 const double *__restrict__ F, double *__restrict__ W, int j0)
{
	const DevFront f = fr[list[blockIdx.x]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0), lane = threadIdx.x;
	double *w = W + f.woff;
	const double *L = F + f.foff;
	double v = lane < nb ? w[j0 + lane] : 0.0;
	long long cb = pk(f.m, j0) + j0; // column j0 + c, row j0
	for (int c = 0; c < nb; ++c)
	{
		const double yc = __shfl_sync(0xffffffffu, v, c) / L[cb + c];
		if (lane == c) v = yc;
		if (lane > c && lane < nb) v = fma(-L[cb + lane], yc, v);
		cb += f.m - (j0 + c) - 1;
	}
	if (lane < nb) w[j0 + lane] = v;
}

__global__ void __launch_bounds__(FWD_ROWS) k_fwd_rows(const DevFront *__restrict__ fr, const int *__restrict__ list,
													   const double *__restrict__ F, double *__restrict__ W, int j0)
{
	const DevFront f = fr[list[blockIdx.y]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0);
	double *w = W + f.woff;
	const double *L = F + f.foff;
	__shared__ double yb[NB];
	if (threadIdx.x < nb) yb[threadIdx.x] = w[j0 + threadIdx.x];
	__syncthreads();
	const long long i = (long long)j0 + nb + (long long)blockIdx.x * FWD_ROWS + threadIdx.x;
	if (i >= f.m) return;
	double a = w[i];
	long long cb = pk(f.m, j0) + i;
	for (int c = 0; c < nb; ++c)
	{
		a = fma(-L[cb], yb[c], a);
		cb += f.m - (j0 + c) - 1;
	}
	w[i] = a;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

// Backward substitution, level by level from the root.  k_bwd_gather: w2 = the
// rows' solution (ancestors, already solved); k_bwd_l21: w1 -= L21^T w2 (a warp
// per column); per panel from the last, k_bwd_cols sums L[i][j] x_i over the
// solved columns i below the panel in row chunks of BWD_ROWS (one partial per
// chunk and column) and k_bwd_diag (one warp per front) adds the partials in chunk
// order and solves the transposed diagonal block in registers; k_bwd_store writes
// x1.
__global__ void __launch_bounds__(256) k_bwd_gather(const DevFront *__restrict__ fr, const int *__restrict__ list,
													const int *__restrict__ rows, const double *__restrict__ X,
													double *__restrict__ W)
{
	const DevFront f = fr[list[blockIdx.x]];
	double *w = W + f.woff;
	const int r = f.m - f.k;
	for (int i = threadIdx.x; i < r; i += 256) w[f.k + i] = X[rows[f.ioff + i]];
}

__global__ void __launch_bounds__(256) k_bwd_l21(const DevFront *__restrict__ fr, const int *__restrict__ list,
												 const double *__restrict__ F, double *__restrict__ W)
{
	const DevFront f = fr[list[blockIdx.y]];
	const int j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
	if (j >= f.k) return;
	double *w = W + f.woff;
	const int r = f.m - f.k;
	const double *Lj = F + f.foff + pk(f.m, j) + f.k;
	double s = 0.0;
	for (int i = lane; i < r; i += 32) s = fma(Lj[i], w[f.k + i], s);
	s = warp_sum_d(s);
	if (lane == 0) w[j] -= s;
}

__global__ void __launch_bounds__(256) k_bwd_cols(const DevFront *__restrict__ fr, const int *__restrict__ list,
												  const double *__restrict__ F, const double *__restrict__ W,
												  double *__restrict__ part, int j0)
{
	const DevFront f = fr[list[blockIdx.y]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0), e = j0 + nb;
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	const double *w = W + f.woff;
	const double *L = F + f.foff;
	const int i0 = e + blockIdx.x * BWD_ROWS, i1 = min(f.k, i0 + BWD_ROWS);
	double *pp = part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * NB;
	for (int c = warp; c < NB; c += 8)
	{
		double s = 0.0;
		if (c < nb)
		{
			const double *Lc = L + pk(f.m, j0 + c);
			for (int i = i0 + lane; i < i1; i += 32) s = fma(Lc[i], w[i], s);
		}
		s = warp_sum_d(s);
		if (lane == 0) pp[c] = s;
	}
}

__global__ void __launch_bounds__(32) k_bwd_diag(const DevFront *__restrict__ fr, const int *__restrict__ list,
												 const double *__restrict__ F, double *__restrict__ W,
												 const double *__restrict__ part, int nchunk, int j0)
{
	const DevFront f = fr[list[blockIdx.x]];
	if (j0 >= f.k) return;
	const int nb = min(NB, f.k - j0), lane = threadIdx.x;
	double *w = W + f.woff;
	const double *L = F + f.foff;
	double v = 0.0;
	if (lane < nb)
	{
		const double *pp = part + (size_t)blockIdx.x * nchunk * NB + lane;
		double s = 0.0;
		for (int q = 0; q < nchunk; ++q) s += pp[(size_t)q * NB];
		v = w[j0 + lane] - s;
	}
	for (int c = nb - 1; c >= 0; --c)
	{
		// x_c = (v_c - sum_{c' > c} L[c'][c] x_c') / L[c][c]; lanes c' > c hold x_c'
		const double *Lc = L + pk(f.m, j0 + c) + j0;
		const double t = lane > c && lane < nb ? Lc[lane] * v : 0.0;
		const double sum = warp_sum_d(t);
		const double xc = (__shfl_sync(0xffffffffu, v, c) - sum) / Lc[c];
		if (lane == c) v = xc;
	}
	if (lane < nb) w[j0 + lane] = v;
}

__global__ void __launch_bounds__(256) k_bwd_store(const DevFront *__restrict__ fr, const int *__restrict__ list,
												   const double *__restrict__ W, double *__restrict__ X)
{
	const DevFront f = fr[list[blockIdx.x]];
	const double *w = W + f.woff;
	for (int j = threadIdx.x; j < f.k; j += 256) X[f.col0 + j] = w[j];
}

} // namespace

// values (device, the analysed pattern's nnz) -> factor; 0 ok, 1 not positive
// definite, else a CUDA error through *ce
int direct_factorize(DirectFactor *f, const double *vals, cudaStream_t s, cudaError_t *ce)
{
	*ce = cudaSuccess;
	f->factorized = false;
	const int nl = (int)f->lvl_start.size() - 1;
	if ((*ce = cudaMemsetAsync(f->d_err, 0, sizeof(int), s)) != cudaSuccess) return 2;
	if ((*ce = cudaFuncSetAttribute(k_dir_syrk64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SYRK64_SMEM)) !=
		cudaSuccess)
		return 2;
	size_t pi = 0;
	for (int h = 0; h < nl; ++h)
	{
		const int nf = f->lvl_start[h + 1] - f->lvl_start[h];
		const int *list = f->d_lvl_list + f->lvl_start[h];
		const long long fb = f->lvl_fbeg[h], fe = f->lvl_fbeg[h + 1];
		if ((*ce = cudaMemsetAsync(f->d_front + fb, 0, 8 * (size_t)(fe - fb), s)) != cudaSuccess) return 2;
		const long long ab = f->lvl_abeg[h], na = f->lvl_abeg[h + 1] - ab;
		if (na > 0)
			k_dir_assemble<<<(unsigned)((na + 255) / 256), 256, 0, s>>>(na, f->d_amap_src + ab, f->d_amap_dst + ab, vals,
																		 f->d_front);
		for (int ci = 0; ci < f->lvl_maxchild[h]; ++ci)
			if (f->lvl_maxrc[h] > 0)
				k_dir_extend_add<<<dim3((f->lvl_maxrc[h] + 7) / 8, nf), 256, 0, s>>>(f->d_fr, list, f->d_child,
																					 f->d_relpos, f->d_front, ci);
		for (; pi < f->fpanels.size() && f->fpanels[pi].lvl == h; ++pi)
		{
			const Panel &p = f->fpanels[pi];
			// panel A
			k_dir_potrf<<<nf, 32, 0, s>>>(f->d_fr, list, f->d_front, p.j0, f->d_err);
			if (p.rows_grid > 0) k_dir_trsm<<<dim3(p.rows_grid, nf), TRSM_ROWS, 0, s>>>(f->d_fr, list, f->d_front, p.j0);
			// A's update of B, then panel B
			if (p.fwd_grid > 0)
			{
				k_dir_panel_update<<<dim3(p.fwd_grid, nf), TRSM_ROWS, 0, s>>>(f->d_fr, list, f->d_front, p.j0);
				k_dir_potrf<<<nf, 32, 0, s>>>(f->d_fr, list, f->d_front, p.j0 + NB, f->d_err);
				if (p.bwd_grid > 0)
					k_dir_trsm<<<dim3(p.bwd_grid, nf), TRSM_ROWS, 0, s>>>(f->d_fr, list, f->d_front, p.j0 + NB);
			}
			if (p.tiles_grid > 0)
				k_dir_syrk64<<<dim3(p.tiles_grid, nf), 256, SYRK64_SMEM, s>>>(f->d_fr, list, f->d_front, p.j0);
		}
		if ((*ce = cudaGetLastError()) != cudaSuccess) return 2;
	}
	int bad = 0;
	if ((*ce = cudaMemcpyAsync(&bad, f->d_err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return 2;
	if ((*ce = cudaStreamSynchronize(s)) != cudaSuccess) return 2;
	if (bad) return 1;
	f->factorized = true;
	return 0;
}

// x = A^-1 b for device vectors b, x of n entries (x may alias b)
cudaError_t direct_solve(DirectFactor *f, const double *b, double *x, cudaStream_t s)
{
	const int n = f->n;
	if (n == 0) return cudaSuccess;
	double *bp = f->d_vec, *xp = f->d_vec + n;
	const int nl = (int)f->lvl_start.size() - 1;
	k_dir_permute_in<<<(n + 255) / 256, 256, 0, s>>>(n, f->d_perm, b, bp);
	size_t pi = 0;
	for (int h = 0; h < nl; ++h)
	{
		const int nf = f->lvl_start[h + 1] - f->lvl_start[h];
		const int *list = f->d_lvl_list + f->lvl_start[h];
		k_fwd_init<<<nf, 256, 0, s>>>(f->d_fr, list, f->d_child, f->d_relpos, bp, f->d_work);
		for (; pi < f->panels.size() && f->panels[pi].lvl == h; ++pi)
		{
			const Panel &p = f->panels[pi];
			k_fwd_diag<<<nf, 32, 0, s>>>(f->d_fr, list, f->d_front, f->d_work, p.j0);
			if (p.fwd_grid > 0)
				k_fwd_rows<<<dim3(p.fwd_grid, nf), FWD_ROWS, 0, s>>>(f->d_fr, list, f->d_front, f->d_work, p.j0);
		}
	}
	for (int h = nl - 1; h >= 0; --h)
	{
		const int nf = f->lvl_start[h + 1] - f->lvl_start[h];
		const int *list = f->d_lvl_list + f->lvl_start[h];
		k_bwd_gather<<<nf, 256, 0, s>>>(f->d_fr, list, f->d_rows, xp, f->d_work);
		if (f->lvl_maxk[h] > 0)
			k_bwd_l21<<<dim3((f->lvl_maxk[h] + 7) / 8, nf), 256, 0, s>>>(f->d_fr, list, f->d_front, f->d_work);
		// this level's panels, last first
		size_t p1 = 0;
		while (p1 < f->panels.size() && f->panels[p1].lvl < h) ++p1;
		size_t p2 = p1;
		while (p2 < f->panels.size() && f->panels[p2].lvl == h) ++p2;
		for (size_t q = p2; q > p1; --q)
		{
			const Panel &p = f->panels[q - 1];
			k_bwd_cols<<<dim3(p.bwd_grid, nf), 256, 0, s>>>(f->d_fr, list, f->d_front, f->d_work, f->d_part, p.j0);
			k_bwd_diag<<<nf, 32, 0, s>>>(f->d_fr, list, f->d_front, f->d_work, f->d_part, p.bwd_grid, p.j0);
		}
		k_bwd_store<<<nf, 256, 0, s>>>(f->d_fr, list, f->d_work, xp);
	}
	k_dir_permute_out<<<(n + 255) / 256, 256, 0, s>>>(n, f->d_perm, xp, x);
	return cudaGetLastError();
}

} // namespace pfg

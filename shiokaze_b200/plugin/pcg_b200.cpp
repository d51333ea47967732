/*
 * pcg_b200.cpp -- Shiokaze linear-solver module backed by the B200 CUDA
 * library (LinSolver=pcg_b200).
 *
 * Drop-in for LinSolver=pcg (src/linsolver/pcg.cpp:32-80): it implements
 * RCMatrix_solver_interface<size_t,double>::solve
 * (include/shiokaze/linsolver/RCMatrix_solver.h:44-77), reads the same keys
 * (Residual, MaxIterations, ModifiedIC, MinDiagRatio) and returns the same
 * Result {count, reresid}. Any projection that solves through an
 * RCMatrix_solver driver (macpressuresolver3, macstreamfuncsolver3, the octree
 * projections) can select it without other changes.
 *
 * The matrix is read row by row through const_for_each, as the reference
 * module reads it into its SparseMatrix (pcg.cpp:47-53): entries of a row
 * are merged by column and kept sorted, so the CSR handed to the GPU equals
 * the reference's FixedSparseMatrix. The GPU runs the algorithm the
 * reference's pcg runs as shipped: conjugate gradients with the identity
 * preconditioner (its MIC(0) result is overwritten,
 * local/include/pcgsolver/pcg_solver.h:379-384), x0 = 0, stopping at
 * ||r||inf <= Residual * ||b||inf, count = iteration + 1, FP64 throughout.
 */
#include <shiokaze/linsolver/RCMatrix_solver.h>
#include <shiokaze/core/console.h>
#include "shkz_b200.h"
#include <algorithm>
#include <cstring>
#include <string>
#include <utility>
#include <vector>
//
SHKZ_USING_NAMESPACE
//
class pcg_b200_solver : public RCMatrix_solver_interface<size_t,double> {
protected:
	//
	LONG_NAME("Conjugate Gradient Solver (B200)")
	ARGUMENT_NAME("PCG")
	//
	virtual ~pcg_b200_solver() {
		if( m_ctx ) shkz_b200_destroy(m_ctx);
	}
	//
	virtual void configure( configuration &config ) override {
		config.get_double("Residual",m_cfg.residual,"Tolerable residual");
		config.get_double("ModifiedIC",m_cfg.mic_omega,"Modified incomplete cholesky");
		config.get_double("MinDiagRatio",m_cfg.mic_min_diag_ratio,"Minimal diagonal ratio");
		unsigned max_it = m_cfg.max_iterations;
		config.get_unsigned("MaxIterations",max_it,"Maximal iteration count");
		m_cfg.max_iterations = max_it;
		int device = m_cfg.device;
		config.get_integer("B200.Device",device,"CUDA device ordinal");
		m_cfg.device = device;
		std::string pre (m_cfg.csr_preconditioner == SHKZ_B200_PRECOND_MIC0 ? "mic0" : "none");
		config.get_string("B200.Preconditioner",pre,"none (as the shipped pcg runs) or mic0 (its MIC(0) applied)");
		m_cfg.csr_preconditioner = pre == "mic0" ? SHKZ_B200_PRECOND_MIC0 : SHKZ_B200_PRECOND_NONE;
	}
	//
	virtual Result solve( const RCMatrix_interface<size_t,double> *A, const RCMatrix_vector_interface<size_t,double> *b,
						  RCMatrix_vector_interface<size_t,double> *x ) const override {
		//
		const size_t n = A->rows();
		std::vector<long long> indptr(n+1,0), indices;
		std::vector<double> data;
		std::vector<std::pair<size_t,double> > row;
		indices.reserve(7*n);
		data.reserve(7*n);
		for( size_t r=0; r<n; ++r ) {
			row.clear();
			A->const_for_each(r,[&]( size_t column, double value ) {
				row.push_back({column,value});
			});
			std::stable_sort(row.begin(),row.end(),[]( const std::pair<size_t,double> &a, const std::pair<size_t,double> &b ) {
				return a.first < b.first;
			});
			for( size_t k=0; k<row.size(); ++k ) {
				if( k && row[k].first == (size_t)indices.back() ) data.back() += row[k].second;
				else {
					indices.push_back((long long)row[k].first);
					data.push_back(row[k].second);
				}
			}
			indptr[r+1] = (long long)indices.size();
		}
		std::vector<double> rhs, result(n,0.0);
		b->convert_to(rhs);
		rhs.resize(n,0.0);
		//
		shkz_b200_result res;
		std::memset(&res,0,sizeof(res));
		int rc = 0;
		if( ! m_ctx ) {
			rc = shkz_b200_create(&m_ctx,&m_cfg);
			if( rc ) m_ctx = nullptr;
		} else {
			shkz_b200_set_config(m_ctx,&m_cfg);
		}
		if( ! rc ) rc = shkz_b200_solve_csr(m_ctx,(long long)n,indptr.data(),indices.data(),data.data(),rhs.data(),result.data(),&res);
		if( rc && rc != SHKZ_B200_ERR_NAN ) {
			console::dump( "pcg_b200: %s (%s)\n", shkz_b200_errstr(rc), m_ctx ? shkz_b200_last_error(m_ctx) : "");
			x->convert_from(std::vector<double>(n,0.0));
			return {0,0.0};
		}
		x->convert_from(result);
		return {(size_t)res.iterations,res.reresid};
	}
	//
	shkz_b200_config m_cfg = make_default_config();
	static shkz_b200_config make_default_config() {
		shkz_b200_config c;
		shkz_b200_default_config(&c);
		c.preconditioner = SHKZ_B200_PRECOND_NONE;
		return c;
	}
	mutable shkz_b200_ctx *m_ctx {nullptr};
};
//
extern "C" module * create_instance() {
	return new pcg_b200_solver();
}
//
extern "C" const char *license() {
	return "MIT";
}

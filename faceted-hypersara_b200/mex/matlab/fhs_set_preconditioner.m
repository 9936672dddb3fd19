function G = fhs_set_preconditioner(G, pU)
% FHS_SET_PRECONDITIONER  Attaches the diagonal preconditioner pU{l}{b} (or
% pU{l}, one vector per channel) of imaging/imaging.m:436-438 to an
% fhs_operator handle.  The data term then takes the ellipsoid projection of
% src/update_dual_data_fidelity.m:126-147, in update_dual_data_fidelity and
% in the solvers (their default non-DR form in the reference).
for l = 1:numel(pU)
    p = pU{l};
    if iscell(p), p = vertcat(p{:}); end
    fhs_mex('measop_set_preconditioner', G.h, l - 1, double(p(:)));
end
G.precond = true;
end

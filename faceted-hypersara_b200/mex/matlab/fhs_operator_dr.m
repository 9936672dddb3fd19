function D = fhs_operator_dr(G)
% FHS_OPERATOR_DR  Visibility-gridding (DR) operator of an fhs_operator
% handle (lib/operators/util_load_data_gen_dr_measurement_operator.m: H = G'G,
% W, Lambda; one block per channel).  Its data entries of channel l are the
% active grid cells; the wrappers accept it wherever they accept G.
D.h = fhs_mex('measop_create_dr', G.h);
D.M = G.M;
D.N = G.N;
D.L = G.L;
D.blocks = cell(G.L, 1);
for l = 1:G.L
    D.blocks{l} = fhs_mex('measop_n_vis', D.h, l - 1);
end
D.channel = 0;
end

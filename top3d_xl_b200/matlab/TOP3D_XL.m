%% Drop-in replacement of TOP3D_XL(inputModel, consType, V0, nLoop, rMin, ...) that runs the
%% optimisation loop on a B200 through the topx_mex gateway (libtopx.so).
%% Same signature, argument checks, console lines and ./out/ files as the reference, including
%% DesignVolume.nii (the padded density volume) and DesignVolume.stl (its 0.5 isosurface with caps).
%% Optional trailing name/value pairs: 'precision', 'fp64' | 'mixed'; 'typeVcycle',
%% 'Adapted' (default, the reference's typeVcycle_) | 'Standard' (FP64 only);
%% 'specifyPassiveRegions', [#LayersBoundary #LayersLoads #LayersFixations] (default [0 0 0]).
function TOP3D_XL(inputModel, consType, V0, nLoop, rMin, varargin)
	precision = 'fp64';
	typeVcycle = 'Adapted';
	passiveRegions = [0 0 0];
	rHat = [];
	args = varargin;
	while numel(args) >= 2 && ischar(args{end-1}) && ...
			any(strcmp(args{end-1}, {'precision', 'typeVcycle', 'specifyPassiveRegions'}))
		switch args{end-1}
			case 'precision', precision = args{end};
			case 'typeVcycle', typeVcycle = args{end};
			otherwise, passiveRegions = args{end};
		end
		args = args(1:end-2);
	end
	switch consType
		case 'GLOBAL'
		case 'LOCAL'
			if 1 ~= numel(args), error('Wrong Input!'); else, rHat = args{1}; end
		otherwise
			return;
	end
	if islogical(inputModel)
		[ny, nx, nz] = size(inputModel);
		if nx < 3 || ny < 3 || nz < 3, error('Inappropriate Input Model!'); end
	end
	outPath = './out/'; if ~exist(outPath, 'dir'), mkdir(outPath); end
	fid = fopen(strcat(outPath, 'RunLog.log'), 'w'); fclose(fid); diary(strcat(outPath, 'RunLog.log'));
	tStartTotal = tic;
	[hist, xPhys, grid] = topx_mex(inputModel, consType, V0, nLoop, rMin, rHat, precision, typeVcycle, ...
		double(passiveRegions));
	disp(['Compliance of Fully Solid Domain: ' sprintf('%16.6e', hist.cSolid)]);
	for loop = 1:numel(hist.c)
		if strcmp(consType, 'GLOBAL')
			fprintf(' It.:%4i Obj.:%16.8e Vol.:%6.4e Sharp.:%6.4e Cons.:%4.2e Ch.:%4.2e\n', ...
				loop, hist.c(loop), hist.vol(loop), hist.sharp(loop), hist.cons(loop), hist.change(loop));
		else
			fprintf(' It.:%4i Obj.:%16.8e Vol.:%6.4e Sharp.:%6.4e Cons.:%4.2e  Ch.:%4.2e \n', ...
				loop, hist.c(loop), hist.vol(loop), hist.sharp(loop), hist.cons(loop), hist.change(loop));
		end
	end
	fid = fopen(strcat(outPath, 'iters_Target.dat'), 'w'); fprintf(fid, '%d\n', hist.its'); fclose(fid);
	fid = fopen(strcat(outPath, 'c_Target.dat'), 'w'); fprintf(fid, '%30.16e\n', hist.c); fclose(fid);
	fid = fopen(strcat(outPath, 'sharp_Target.dat'), 'w'); fprintf(fid, '%30.16e\n', hist.sharp); fclose(fid);
	fid = fopen(strcat(outPath, 'timing_Target.dat'), 'w'); fprintf(fid, '%16.6e\n', hist.tTotal); fclose(fid);
	V = zeros(grid.resX * grid.resY * grid.resZ, 1);
	V(double(grid.eleMapBack)) = xPhys;
	V = reshape(V, grid.resY, grid.resX, grid.resZ);
	topx_mex('write_design', V, outPath);   % DesignVolume.nii and DesignVolume.stl
	disp(['..........Performing Topology Optimization Costs (in total): ', sprintf('%10.4e', toc(tStartTotal)), 's.']);
	diary off;
end
